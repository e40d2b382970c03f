// Internal definitions shared by the batch C ABI (capi.cu) and the serving
// engine (serve.cu): the device-resident batch and the operations on it.
//
// A batch's VDF state is a block list per cell (global IDs, slot = offset and
// count into the list) plus, optionally, a per-block index into the data pool
// that holds the values.  Sweeps are out of place between two data pools and
// leave a direct state (block b of a cell is data row off+b).  Block
// adjustment leaves an indirect state (a new list whose entries point at the
// kept rows, or at no row for added zero blocks), so it moves no VDF data.
//
// The acceleration transform's pivot (the first moments of the current VDF)
// sits in its own record; pivot_valid says it describes the current state.
// Every change of the state clears it (set_direct_state, adjustment,
// materialisation, serving admissions), and the single-read moments that end
// an acceleration step or compute the Vlasov step's "_R" moments set it, so
// the next step skips its separate first-moments pass.
#pragma once
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <vector>

#include "vlgpu_common.cuh"

namespace vlgpu {
cudaError_t launch_rebase_work(SweepCounters* counters, cudaStream_t stream);
cudaError_t launch_columnize(int dim, const uint32_t* gids, const uint32_t* src_index, const CellSlot* src_slots,
                             CellSlot* dst_slots, uint32_t* perm, ColumnSet* sets, uint32_t set_capacity,
                             uint32_t dst_capacity, const SweepCell* sweep_cells, uint32_t* status,
                             SweepCounters* counters, BatchStats* stats, const MeshDev& mesh, int wall_margin,
                             uint32_t cell_begin, uint32_t cell_end, int first_of_step, cudaStream_t stream);
cudaError_t launch_columnize_batch(int dim, const uint32_t* gids, const uint32_t* src_index,
                                   const CellSlot* src_slots, CellSlot* dst_slots, uint32_t* perm, ColumnSet* sets,
                                   uint32_t set_capacity, uint32_t dst_capacity, const SweepCell* sweep_cells,
                                   uint32_t* status, SweepCounters* counters, BatchStats* stats, const MeshDev& mesh,
                                   int wall_margin, uint32_t n_cells, int first_of_step, uint32_t* wide_cells,
                                   const uint32_t* order, int wide_grid, cudaStream_t stream);
int columnize_wide_blocks_per_sm(const MeshDev& mesh);
cudaError_t launch_remap(int dim, const ColumnSet* sets, SweepCounters* counters, const uint32_t* perm,
                         const float* src_data, float* dst_data, uint32_t* dst_gids, const SweepCell* sweep_cells,
                         uint32_t* status, const MeshDev& mesh, int wall_margin, uint32_t set_capacity,
                         uint8_t* content_out, double content_threshold, bool exact, int recon, int grid,
                         cudaStream_t stream);
int remap_blocks_per_sm();
struct CellAccelInputs {
   double B[3];
   double curl[3];
   double egradpe[3];
   double dt;
};
cudaError_t launch_moments(const uint32_t* gids, const uint32_t* src_index, const float* data, const CellSlot* slots,
                           double* moments, const double* shift, const MeshDev& mesh, const double vmin[3],
                           const double bs[3], const double dv[3], double mass, double charge, bool second,
                           uint32_t n_cells, double* part_sums, uint32_t* done, int grid, cudaStream_t stream);
cudaError_t launch_moments_both(const uint32_t* gids, const uint32_t* src_index, const float* data,
                                const CellSlot* slots, double* pivot, double* moments, const MeshDev& mesh,
                                const double vmin[3], const double bs[3], const double dv[3], double mass,
                                double charge, uint32_t n_cells, double* part_sums, uint32_t* done, int grid,
                                cudaStream_t stream);
int moments_blocks_per_sm();
cudaError_t launch_geometry(const CellAccelInputs* in, const double* moments, double* isect12, SweepCell* sweep3,
                            uint32_t n_cells, double q, double m, double hall_min_rhoq, int ohm_gradpe, double mu0,
                            const double vmin[3], const double dv[3], uint32_t map_order, float threshold,
                            cudaStream_t stream);
cudaError_t launch_adjust(const uint32_t* gids, const uint32_t* src_index, const CellSlot* slots,
                          const uint8_t* content, const float* data, const int32_t* neighbors, uint32_t* out_gids,
                          uint32_t* out_src,
                          CellSlot* out_slots, double* loss, uint32_t* status, SweepCounters* counters,
                          uint32_t out_capacity, const MeshDev& mesh, double min_value, int add_width, double dv3,
                          uint32_t n_cells, uint32_t* scratch, int grid, const uint32_t* order, MaskRec* masks,
                          uint32_t* pool, uint32_t* pool_top, uint32_t pool_cap, double* mom_record,
                          double* pivot, int write_pivot, const MomentFrame& frame, cudaStream_t stream);
int adjust_blocks_per_sm();
size_t adjust_scratch_words(const MeshDev& mesh);
cudaError_t launch_max_dt(const uint32_t* gids, const CellSlot* slots, const CellAccelInputs* in, const MeshDev& mesh,
                          const double vmin[3], const double bs[3], const double dv[3], const double dx[3], double q,
                          double m, double max_rotation_deg, double* r_dt, double* v_dt, uint32_t n_cells,
                          cudaStream_t stream);
struct FillCell {
   double n;
   double T[3];
   double frame[9];
   double V[3];
   int lo[3], hi[3];
   uint32_t row;
   uint32_t isotropic;
};
cudaError_t launch_fill(const FillCell* cells, uint32_t n_cells, const MeshDev& mesh, const double vmin[3],
                        const double bs[3], const double dv[3], double mass, uint32_t* gids, float* data,
                        CellSlot* slots, cudaStream_t stream);
cudaError_t launch_materialize(const uint32_t* src_index, const float* src, float* dst, uint64_t n_blocks,
                               cudaStream_t stream);
cudaError_t launch_slots_to_host(const CellSlot* src, CellSlot* host_dst, uint32_t n, cudaStream_t stream);
cudaError_t launch_materialize_rows(const uint32_t* src_index, const float* src, float* dst, const uint32_t* n_rows,
                                    int grid, cudaStream_t stream);
struct TransCounters {
   uint32_t n_items;
   uint32_t work;
   uint32_t overflow;
   uint32_t pad;
};
constexpr uint32_t TR_MAX_N = 128;
cudaError_t launch_pencil_union(const uint32_t* gids, const CellSlot* slots, int dim, uint32_t nx, uint32_t ny,
                                uint32_t nz, const MeshDev& mesh, uint32_t* item_gid, uint32_t* item_pencil,
                                uint32_t* rows, uint32_t* srcs, const uint32_t* src_index, uint32_t item_cap,
                                uint64_t row_cap, TransCounters* tc, uint32_t* status, cudaStream_t stream);
cudaError_t launch_trans_remap(int dim, uint32_t N, const uint32_t* item_gid, const uint32_t* item_pencil,
                               const uint32_t* rows, const uint32_t* srcs, TransCounters* tc, uint32_t item_cap,
                               uint64_t row_cap, const uint32_t* src_index, const float* src, float* dst,
                               uint32_t* dst_gids, const MeshDev& mesh, float dt, float dz, float threshold, bool exact,
                               int grid, cudaStream_t stream);
int trans_blocks_per_sm(uint32_t N, bool exact);
uint32_t union_words(const MeshDev& mesh);
constexpr int MOM_COUNT = 16;
constexpr double MU_0 = 1.25663706e-6;  // physicalconstants::MU_0 (common.h:561)
}  // namespace vlgpu

using namespace vlgpu;

struct vlgpu_batch {
   int device = 0;
   vlgpu_mesh mesh{};
   vlgpu_params params{};
   MeshDev mdev{};
   uint32_t n_cells = 0;
   uint64_t capacity = 0;  // blocks per pool
   cudaStream_t stream = nullptr;
   int sm_count = 0;
   int remap_grid = 0;
   // launch shapes in CTAs per SM (0 = occupancy maximum): remap, moments,
   // adjustment, translation; their maxima; whether the caller pinned them
   uint32_t cps[4] = {0, 0, 0, 0};
   int cps_max[4] = {0, 0, 0, 0};
   bool launch_pinned = false;
   char device_name[256] = {0};  // the key of the launch tuning table
   bool exact = false;  // remap arithmetic: false = fused, true = the reference's operation order
   int recon = 2;       // acceleration reconstruction: 1 PLM, 2 PPM, 4 PQM
   double vmin_d[3], bs_d[3], dv_d[3];
   // data pools and the lists written by sweeps into them
   uint32_t* gids[2] = {nullptr, nullptr};
   float* data[2] = {nullptr, nullptr};
   CellSlot* slots[2] = {nullptr, nullptr};
   uint8_t* content = nullptr;  // content flag per output row of the last sweep
   // lists written by block adjustment (two, used alternately)
   uint32_t* adj_gids[2] = {nullptr, nullptr};
   uint32_t* adj_src[2] = {nullptr, nullptr};
   CellSlot* adj_slots[2] = {nullptr, nullptr};
   int adj_next = 0;
   // rows in use: [0], [1] data pools (and their sweep lists), [2], [3] the
   // adjustment lists; device copies of the allocation counters
   uint32_t* rows_used = nullptr;
   int st_list = 0;  // which rows_used entry describes the current list
   // the current state
   const uint32_t* st_gids = nullptr;
   const uint32_t* st_src = nullptr;  // null: direct
   const CellSlot* st_slots = nullptr;
   int cur = 0;                       // data pool holding the values
   bool content_valid = false;        // content[] describes the current list
   bool pivot_valid = false;          // pivot holds the first moments of the current VDF
   // work arrays
   uint32_t* perm = nullptr;
   ColumnSet* sets = nullptr;
   SweepCell* sweep_cells = nullptr;
   SweepCell* sweep3 = nullptr;  // 3 * n_cells, from the device geometry
   CellAccelInputs* accel_in = nullptr;
   double* moments = nullptr;  // MOM_COUNT per cell
   double* pivot = nullptr;    // MOM_COUNT per cell: first moments (U = 0) the acceleration transform uses
   double* mom_scratch = nullptr;  // MOM_COUNT per cell: a record for pivots of some cells only
   double* mom_parts = nullptr;   // per cell and part, the part's sums (moments work array)
   uint32_t* mom_done = nullptr;  // per cell, the parts finished (zero between passes)
   int mom_grid = 0;
   double* isect12 = nullptr;  // 12 per cell
   double* loss = nullptr;     // RHOLOSSADJUST per cell
   uint32_t* status = nullptr;
   SweepCounters* counters = nullptr;
   BatchStats* stats = nullptr;
   // spatial grid (uniform, periodic, cells x fastest) and translation work arrays
   bool has_grid = false;
   uint32_t grid_dims[3] = {0, 0, 0};
   double grid_dx[3] = {0.0, 0.0, 0.0};
   uint32_t* item_gid = nullptr;
   uint32_t* item_pencil = nullptr;
   uint32_t* trans_rows = nullptr;  // per item and pencil cell: list row of the block (or none)
   uint32_t* trans_src = nullptr;   // the same entries: data index in the source pool (or none)
   uint64_t row_cap = 0;
   TransCounters* tcounters = nullptr;
   int32_t* neighbors = nullptr;  // 26 per cell (-1: none), the spatial neighbours block adjustment consults
   double* dt_buf = nullptr;      // 2 per cell: r-space and v-space time-step limits
   uint32_t* adj_scratch = nullptr;  // per adjustment CTA: masks of a cell too wide for shared memory
   uint32_t* wide_cells = nullptr;  // the cells whose columnize plane is too wide for the capped kernel
   uint32_t* cell_order = nullptr;  // the cells by decreasing block count at the last upload (persistent kernels)
   uint32_t* h_order = nullptr;     // pinned staging of cell_order
   uint32_t* halo_scratch = nullptr;  // cell descriptors of a pack / unpack of some cells (grown on demand)
   size_t halo_words = 0;
   vlgpu::MaskRec* mask_recs = nullptr;  // grid: per cell, its content mask record
   uint32_t* mask_pool = nullptr;        // grid: the content mask rows
   uint32_t* mask_top = nullptr;         // grid: words of the pool in use
   uint32_t mask_cap = 0;
   int adj_grid = 0;
   int col_wide_grid = 0;  // CTAs of the wide-plane columnize
   double* moments_r = nullptr;   // MOM_COUNT per cell: the moments after translation (the "_R" set)
   // pinned staging; each buffer's event marks when its last copy was read
   SweepCell* h_sweep = nullptr;
   CellAccelInputs* h_accel = nullptr;
   vlgpu::CellSlot* h_slots_in = nullptr;   // n_cells slots and the row count of an asynchronous upload
   vlgpu::CellSlot* h_slots_out = nullptr;  // n_cells slots of an asynchronous download (mapped pinned)
   vlgpu::CellSlot* d_slots_out = nullptr;  // its device address
   cudaEvent_t ev_sweep = nullptr, ev_accel = nullptr, ev_upload = nullptr, ev_slots = nullptr;
   cudaEvent_t ev_order = nullptr;  // the last copy of h_order
   // captured step sequences (vlgpu_batch_capture): the executable graph and
   // the buffer state it starts and ends in
   struct GraphSlot {
      cudaGraphExec_t exec = nullptr;
      const uint32_t* st_gids = nullptr;
      const uint32_t* st_src = nullptr;
      const vlgpu::CellSlot* st_slots = nullptr;
      int cur = 0;
      int adj_next = 0;
      bool pivot_valid = false;      // at the start of the captured steps
      bool pivot_valid_end = false;  // after them
      unsigned long long launches = 0;
      unsigned long long remap_launches = 0;
   };
   GraphSlot graphs[8];
   // host-side accounting
   unsigned long long launches = 0;
   unsigned long long remap_launches = 0;
   bool profiling = false;
   std::vector<cudaEvent_t> prof_events;
   size_t prof_used = 0;
};

namespace vlgpu_batch_ops {

int cuda_status(cudaError_t e, const char* what);

#define VL_CHECK(call)                                          \
   do {                                                         \
      int _s = vlgpu_batch_ops::cuda_status((call), #call);     \
      if (_s != VLGPU_OK) return _s;                            \
   } while (0)

void free_batch(vlgpu_batch* b);
void set_direct_state(vlgpu_batch* b, int pool);
int sweep_device(vlgpu_batch* b, const vlgpu::SweepCell* sweep_cells, uint32_t dim, bool per_cell, bool first_of_step);
int moments_device(vlgpu_batch* b, bool second, double* record = nullptr, const double* shift = nullptr);
int moments_both_device(vlgpu_batch* b, double* record);
int adjust_device(vlgpu_batch* b, double* record = nullptr, bool write_pivot = false);
int materialize(vlgpu_batch* b);
int materialize_async(vlgpu_batch* b);
int geometry_device(vlgpu_batch* b, uint32_t map_order);
int accelerate_device(vlgpu_batch* b, uint32_t map_order, bool per_cell, bool next_pivot = true);
int translate_device(vlgpu_batch* b, uint32_t dim, double dt);
int stage_fields(vlgpu_batch* b, const vlgpu_cell_fields* fields, const double* dt);
int vlasov_step_device(vlgpu_batch* b, double dt, uint32_t map_order);
void apply_launch(vlgpu_batch* b);
void consult_launch_table(vlgpu_batch* b, double mean_blocks);

}  // namespace vlgpu_batch_ops
