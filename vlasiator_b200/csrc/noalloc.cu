// vlgpu_map_1d_noalloc: the SLICE-3D 1D sweep for callers that must not
// allocate device memory.
//
// Who needs it: a host code that reserves all of the GPU's memory for its own
// pool allocator at start-up (so a cudaMalloc from a library either fails or
// breaks that budget), and a code that calls the sweep on a latency-critical
// path where cudaMalloc/cudaFree would synchronise the whole device and stall
// its other streams.  Such a caller can hold its blocks in its own device
// buffers but cannot let vlgpu_batch_create allocate pools and work arrays.
//
// The sweep's work arrays (per-cell slots and sweep parameters, the source
// permutation, the column sets, the counters and the per-block content flags)
// live here in one file-scope device array of fixed size, which every GPU
// that loads libvlgpu.so keeps until the process exits.  The kernels are the
// ones vlgpu_map_1d launches with its default (fused PPM) arithmetic; only the
// place of their work arrays differs.
#include <cstddef>
#include <cstdio>
#include <mutex>

#include "vlgpu_common.cuh"

namespace vlgpu {
cudaError_t launch_columnize(int dim, const uint32_t* gids, const uint32_t* src_index, const CellSlot* src_slots,
                             CellSlot* dst_slots, uint32_t* perm, ColumnSet* sets, uint32_t set_capacity,
                             uint32_t dst_capacity, const SweepCell* sweep_cells, uint32_t* status,
                             SweepCounters* counters, BatchStats* stats, const MeshDev& mesh, int wall_margin,
                             uint32_t cell_begin, uint32_t cell_end, int first_of_step, cudaStream_t stream);
cudaError_t launch_remap(int dim, const ColumnSet* sets, SweepCounters* counters, const uint32_t* perm,
                         const float* src_data, float* dst_data, uint32_t* dst_gids, const SweepCell* sweep_cells,
                         uint32_t* status, const MeshDev& mesh, int wall_margin, uint32_t set_capacity,
                         uint8_t* content_out, double content_threshold, bool exact, int recon, int grid,
                         cudaStream_t stream);
int remap_blocks_per_sm();

namespace {

constexpr uint32_t NA_MAX_BLOCKS = VLGPU_NOALLOC_MAX_BLOCKS;
constexpr uint32_t NA_MAX_CELLS = VLGPU_NOALLOC_MAX_CELLS;
constexpr int NA_MAX_DEVICES = 64;

// Layout of the scratch array.  Everything up to `zeroed_end` is cleared at
// the start of every call; the rest is fully written before it is read.
struct NoallocLayout {
   SweepCounters counters;
   uint32_t bad_gid;
   uint32_t pad0[3];
   BatchStats stats;
   uint32_t status[NA_MAX_CELLS];
   unsigned char zeroed_end[16];
   CellSlot src_slots[NA_MAX_CELLS];
   CellSlot dst_slots[NA_MAX_CELLS];
   SweepCell sweep[NA_MAX_CELLS];
   uint32_t perm[NA_MAX_BLOCKS];
   ColumnSet sets[NA_MAX_BLOCKS];   // a column set holds at least one source block
   uint8_t content[NA_MAX_BLOCKS];  // written by the remap for every output block
};

// The scratch itself (about 3.3 MB).  In host code this name is only a
// stand-in for the device variable: its device address comes from
// cudaGetSymbolAddress, on every call.
static __device__ __align__(256) unsigned char noalloc_scratch[sizeof(NoallocLayout)];

struct DeviceSetup {
   bool ready;
   int remap_grid;
};
std::mutex setup_mutex;
DeviceSetup setups[NA_MAX_DEVICES];

int na_status(cudaError_t e, const char* what) {
   if (e == cudaSuccess) return VLGPU_OK;
   std::fprintf(stderr, "vlgpu_map_1d_noalloc: %s: %s\n", what, cudaGetErrorString(e));
   return VLGPU_ECUDA;
}

#define NA_CHECK(call)                      \
   do {                                     \
      int _s = na_status((call), #call);    \
      if (_s != VLGPU_OK) return _s;        \
   } while (0)

// Set-up of every call, with the calling device current: the device address
// of noalloc_scratch (looked up each time, so that a context that was
// destroyed and created again after an earlier call is served at the
// scratch's new address) and, once per device, the remap grid size.
int setup_device(int dev, unsigned char** base, int* remap_grid) {
   void* ptr = nullptr;
   NA_CHECK(cudaGetSymbolAddress(&ptr, noalloc_scratch));
   *base = static_cast<unsigned char*>(ptr);
   std::lock_guard<std::mutex> lock(setup_mutex);
   DeviceSetup& s = setups[dev];
   if (!s.ready) {
      int sms = 0;
      NA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      s.remap_grid = sms * remap_blocks_per_sm();
      s.ready = true;
   }
   *remap_grid = s.remap_grid;
   return VLGPU_OK;
}

// Flags any block ID outside the mesh; the sweep kernels index shared memory
// by the block coordinates and must not see one.
__global__ void check_gids_kernel(const uint32_t* __restrict__ gids, uint64_t begin, uint64_t end, uint32_t max_gid,
                                  uint32_t* __restrict__ bad) {
   for (uint64_t q = begin + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < end;
        q += (uint64_t)gridDim.x * blockDim.x)
      if (gids[q] >= max_gid) atomicOr(bad, 1u);
}

}  // namespace
}  // namespace vlgpu

using namespace vlgpu;

extern "C" int vlgpu_map_1d_noalloc(const vlgpu_mesh* mesh, const vlgpu_params* params, uint32_t n_cells,
                                    const uint64_t* offsets, const uint32_t* gids_in, const float* data_in,
                                    const double* intersections, uint32_t dimension, uint32_t* gids_out,
                                    float* data_out, uint64_t out_capacity, uint32_t* cell_off, uint32_t* cell_count,
                                    uint32_t* status, void* stream) {
   if (!mesh || !params || !offsets || !intersections || !cell_off || !cell_count || dimension > 2) return VLGPU_EINVAL;
   if (n_cells == 0 || n_cells > NA_MAX_CELLS) {
      std::fprintf(stderr, "vlgpu_map_1d_noalloc: %u cells requested, the limit is 1..%u cells per call\n", n_cells,
                   NA_MAX_CELLS);
      return VLGPU_EINVAL;
   }
   for (int d = 0; d < 3; ++d)
      if (mesh->len[d] == 0 || mesh->len[d] > (uint32_t)MAX_LEN || !(mesh->vmax[d] > mesh->vmin[d]))
         return VLGPU_EINVAL;
   if (!(params->min_value > 0.0)) return VLGPU_EINVAL;
   for (uint32_t c = 0; c < n_cells; ++c)
      if (offsets[c + 1] < offsets[c]) return VLGPU_EINVAL;
   const uint64_t begin = offsets[0], end = offsets[n_cells];
   if (end > NA_MAX_BLOCKS) {
      std::fprintf(stderr,
                   "vlgpu_map_1d_noalloc: input blocks reach index %llu, the limit is %u blocks per call "
                   "(offsets[n_cells] <= %u)\n",
                   (unsigned long long)end, NA_MAX_BLOCKS, NA_MAX_BLOCKS);
      return VLGPU_EINVAL;
   }
   if (end > begin && (!gids_in || !data_in)) return VLGPU_EINVAL;
   if (out_capacity > 0 && (!gids_out || !data_out)) return VLGPU_EINVAL;
   if (end > begin && ((const void*)data_out == (const void*)data_in || (const void*)gids_out == (const void*)gids_in)) {
      std::fprintf(stderr, "vlgpu_map_1d_noalloc: the output buffers must not be the input buffers\n");
      return VLGPU_EINVAL;
   }
   if ((reinterpret_cast<uintptr_t>(data_in) | reinterpret_cast<uintptr_t>(data_out)) & 15u) {
      std::fprintf(stderr, "vlgpu_map_1d_noalloc: data_in and data_out must be 16-byte aligned\n");
      return VLGPU_EINVAL;
   }

   int dev = 0;
   NA_CHECK(cudaGetDevice(&dev));
   if (dev < 0 || dev >= NA_MAX_DEVICES) return VLGPU_ENODEV;
   unsigned char* base = nullptr;  // device address of noalloc_scratch on this device
   int remap_grid = 0;
   const int st = setup_device(dev, &base, &remap_grid);
   if (st != VLGPU_OK) return st;
   cudaStream_t s = static_cast<cudaStream_t>(stream);

   // device views of the scratch
   SweepCounters* d_counters = reinterpret_cast<SweepCounters*>(base + offsetof(NoallocLayout, counters));
   uint32_t* d_bad = reinterpret_cast<uint32_t*>(base + offsetof(NoallocLayout, bad_gid));
   BatchStats* d_stats = reinterpret_cast<BatchStats*>(base + offsetof(NoallocLayout, stats));
   uint32_t* d_status = reinterpret_cast<uint32_t*>(base + offsetof(NoallocLayout, status));
   CellSlot* d_src_slots = reinterpret_cast<CellSlot*>(base + offsetof(NoallocLayout, src_slots));
   CellSlot* d_dst_slots = reinterpret_cast<CellSlot*>(base + offsetof(NoallocLayout, dst_slots));
   SweepCell* d_sweep = reinterpret_cast<SweepCell*>(base + offsetof(NoallocLayout, sweep));
   uint32_t* d_perm = reinterpret_cast<uint32_t*>(base + offsetof(NoallocLayout, perm));
   ColumnSet* d_sets = reinterpret_cast<ColumnSet*>(base + offsetof(NoallocLayout, sets));
   uint8_t* d_content = reinterpret_cast<uint8_t*>(base + offsetof(NoallocLayout, content));

   // host staging on the stack (no heap use either)
   SweepCell h_sweep[NA_MAX_CELLS];
   CellSlot h_slots[NA_MAX_CELLS];
   uint32_t h_status[NA_MAX_CELLS];
   for (uint32_t c = 0; c < n_cells; ++c) {
      h_sweep[c] = make_sweep_cell(intersections + 4 * (size_t)c, dimension, params->min_value);
      h_slots[c].off = (uint32_t)offsets[c];
      h_slots[c].count = (uint32_t)(offsets[c + 1] - offsets[c]);
   }
   MeshDev mdev{};
   for (int d = 0; d < 3; ++d) {
      const double bs = (mesh->vmax[d] - mesh->vmin[d]) / mesh->len[d];
      mdev.len[d] = mesh->len[d];
      mdev.dv[d] = (float)(bs / WID);
      mdev.vmin[d] = (float)mesh->vmin[d];
   }

   // the previous call's counters, flags and statuses must not leak into this one
   NA_CHECK(cudaMemsetAsync(base, 0, offsetof(NoallocLayout, zeroed_end), s));
   NA_CHECK(cudaMemcpyAsync(d_sweep, h_sweep, sizeof(SweepCell) * n_cells, cudaMemcpyHostToDevice, s));
   NA_CHECK(cudaMemcpyAsync(d_src_slots, h_slots, sizeof(CellSlot) * n_cells, cudaMemcpyHostToDevice, s));
   if (end > begin) {
      uint32_t h_bad = 0;
      const uint32_t max_gid = mesh->len[0] * mesh->len[1] * mesh->len[2];
      const uint64_t n = end - begin;
      const unsigned grid = (unsigned)((n + 255) / 256 < 1024 ? (n + 255) / 256 : 1024);
      check_gids_kernel<<<grid, 256, 0, s>>>(gids_in, begin, end, max_gid, d_bad);
      NA_CHECK(cudaGetLastError());
      NA_CHECK(cudaMemcpyAsync(&h_bad, d_bad, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      NA_CHECK(cudaStreamSynchronize(s));
      if (h_bad) {
         std::fprintf(stderr, "vlgpu_map_1d_noalloc: a block ID lies outside the %u-block mesh\n", max_gid);
         return VLGPU_EINVAL;
      }
   }

   const uint32_t dst_cap = (uint32_t)(out_capacity < NA_MAX_BLOCKS ? out_capacity : NA_MAX_BLOCKS);
   const int wm = (int)params->wall_margin;
   NA_CHECK(launch_columnize((int)dimension, gids_in, nullptr, d_src_slots, d_dst_slots, d_perm, d_sets,
                             NA_MAX_BLOCKS, dst_cap, d_sweep, d_status, d_counters, d_stats, mdev, wm, 0, n_cells, 0,
                             s));
   NA_CHECK(launch_remap((int)dimension, d_sets, d_counters, d_perm, data_in, data_out, gids_out, d_sweep, d_status,
                         mdev, wm, NA_MAX_BLOCKS, d_content, params->min_value, false, 2, remap_grid, s));

   SweepCounters h_counters{};
   NA_CHECK(cudaMemcpyAsync(h_slots, d_dst_slots, sizeof(CellSlot) * n_cells, cudaMemcpyDeviceToHost, s));
   NA_CHECK(cudaMemcpyAsync(h_status, d_status, sizeof(uint32_t) * n_cells, cudaMemcpyDeviceToHost, s));
   NA_CHECK(cudaMemcpyAsync(&h_counters, d_counters, sizeof(SweepCounters), cudaMemcpyDeviceToHost, s));
   NA_CHECK(cudaStreamSynchronize(s));
   for (uint32_t c = 0; c < n_cells; ++c) {
      cell_off[c] = h_slots[c].off;
      cell_count[c] = h_slots[c].count;
      if (status) status[c] = h_status[c];
   }
   if (h_counters.overflow) {
      std::fprintf(stderr, "vlgpu_map_1d_noalloc: the output needs more than %u blocks (out_capacity %llu, limit %u)\n",
                   dst_cap, (unsigned long long)out_capacity, NA_MAX_BLOCKS);
      return VLGPU_ENOMEM;
   }
   return VLGPU_OK;
}
