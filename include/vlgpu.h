/*
 * vlgpu.h -- C ABI of the B200 Vlasov hot path (libvlgpu.so).
 *
 * The entry points act on a device-resident batch of spatial cells, each
 * holding one population's sparse velocity mesh: a list of velocity-block
 * global IDs (GID = i + j*Nx + k*Nx*Ny) and 64 Realf (float) values per
 * block, x fastest.  They replace, for that data, the reference's
 * per-cell CPU functions listed beside each declaration (paths relative to
 * the Vlasiator source tree).  Plain pointers and sizes only; all calls
 * return a VLGPU_* status code.  A batch belongs to one host thread at a time.
 */
#ifndef VLGPU_H
#define VLGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  Per-cell conditions are also reported bitwise through
   vlgpu_batch_status (VLGPU_CELL_*). */
#define VLGPU_OK 0
#define VLGPU_EINVAL 1    /* bad argument */
#define VLGPU_ENOMEM 2    /* device allocation failed or a pool is full */
#define VLGPU_EWALL 3     /* some target block came within the wall margin (reference bail-out, cpu_acc_map.cpp:325-338) */
#define VLGPU_ETIMEDOUT 4 /* a bounded device-side wait gave up */
#define VLGPU_ERANGE 5    /* a column's target window exceeded the remap ring (rotation per step too large) */
#define VLGPU_ECUDA 6     /* CUDA runtime error */
#define VLGPU_ENODEV 7    /* no CUDA device */
#define VLGPU_EAGAIN 8    /* a served request has not finished yet */
#define VLGPU_ENOENT 9    /* no entry (the launch table has none for the device) */

#define VLGPU_CELL_WALL 1u
#define VLGPU_CELL_RANGE 2u
#define VLGPU_CELL_NOMEM 4u
#define VLGPU_CELL_BADDK 8u

/* Velocity mesh: vmesh::MeshParameters (velocity_mesh_parameters.h:53).
   len = blocks per axis (<= 96); WID = 4 cells per block per axis. */
typedef struct vlgpu_mesh {
   double vmin[3];
   double vmax[3];
   uint32_t len[3];
} vlgpu_mesh;

/* Species and solver settings read by the hot path
   (object_wrapper.cpp:44-68,111-145; parameters.cpp:392-493). */
typedef struct vlgpu_params {
   double charge;            /* C */
   double mass;              /* kg */
   double min_value;         /* <pop>_sparse.minValue */
   uint32_t add_width_v;     /* <pop>_sparse.blockAddWidthV */
   uint32_t wall_margin;     /* bailout.velocity_space_wall_block_margin */
   double hall_minimum_rhoq; /* Parameters::hallMinimumRhoq */
   uint32_t ohm_gradpe;      /* fieldsolver.ohmGradPeTerm */
   uint32_t reserved;
} vlgpu_params;

/* Per-cell field inputs of the acceleration transform, as read from
   SpatialCell::parameters / derivativesBVOL (cpu_acc_transform.cpp:71-89). */
typedef struct vlgpu_cell_fields {
   double B[3];       /* BGB?VOL + PERB?VOL */
   double curl[3];    /* (dBZdy - dBYdz, dBXdz - dBZdx, dBYdx - dBXdy) of the perturbed field */
   double egradpe[3]; /* E?GRADPE; RHOQ_V and V_V come from the cell's own moments */
} vlgpu_cell_fields;

typedef struct vlgpu_batch vlgpu_batch;

/* ---- batch life cycle ---------------------------------------------------- */

/* Creates a batch of n_cells cells on `device` with room for block_capacity
   blocks per pool (two pools are kept for out-of-place sweeps). */
int vlgpu_batch_create(const vlgpu_mesh* mesh, const vlgpu_params* params, uint32_t n_cells, uint64_t block_capacity,
                       int device, vlgpu_batch** out);
int vlgpu_batch_destroy(vlgpu_batch* b);

/* Host -> device: cell c owns blocks offsets[c] .. offsets[c+1]-1 of gids /
   data (64 floats per block).  Replaces the blocks of every cell and clears
   the per-cell status. */
int vlgpu_batch_upload(vlgpu_batch* b, const uint64_t* offsets, const uint32_t* gids, const float* data);

/* Number of blocks per cell (n_cells entries). */
int vlgpu_batch_block_counts(vlgpu_batch* b, uint32_t* counts);

/* Device -> host: blocks of every cell, ascending GID within a cell, packed
   by cell; offsets has n_cells+1 entries; capacity in blocks. */
int vlgpu_batch_download(vlgpu_batch* b, uint64_t* offsets, uint32_t* gids, float* data, uint64_t capacity);

/* Device -> host without reordering: the pool holding the current state is
   copied verbatim up to its highest used block (*used blocks); cell c owns
   blocks cell_off[c] .. cell_off[c]+cell_count[c]-1 of it, in the sweep's
   output order (like the reference's local-ID order, not sorted). */
int vlgpu_batch_download_raw(vlgpu_batch* b, uint32_t* cell_off, uint32_t* cell_count, uint32_t* gids, float* data,
                             uint64_t capacity, uint64_t* used);

/* Asynchronous forms of upload and download_raw for pipelines of several
   batches (no reference counterpart).  vlgpu_batch_upload_async does the
   same checks as vlgpu_batch_upload but only enqueues the copies: gids and
   data (pinned host memory for overlap) must stay untouched until the
   batch's work is done (vlgpu_batch_sync).  vlgpu_batch_download_begin
   enqueues the compaction of an adjusted state and the copy of the cell
   slots; vlgpu_batch_download_end waits for those slots only, fills cell_off,
   cell_count and *used as vlgpu_batch_download_raw does and enqueues the
   copy of gids and data, which hold the result after vlgpu_batch_sync. */
int vlgpu_batch_upload_async(vlgpu_batch* b, const uint64_t* offsets, const uint32_t* gids, const float* data);
int vlgpu_batch_download_begin(vlgpu_batch* b);
int vlgpu_batch_download_end(vlgpu_batch* b, uint32_t* cell_off, uint32_t* cell_count, uint32_t* gids, float* data,
                             uint64_t capacity, uint64_t* used);

/* Ghost-cell exchange of a spatial grid split over several batches (one per
   GPU and rank).  No reference counterpart as an entry point: this is the
   data movement of the remote-neighbour updates of a distributed grid
   (update_remote_mapping_contribution_amr, vlasovsolver/cpu_trans_map_amr.cpp:
   493-810, and dccrg's neighbour-data updates), rebuilt as a pack into a
   device buffer, a transfer the caller makes (NCCL send/recv or any other)
   and an unpack into the receiving batch.  Both return after their device
   work is done.

   vlgpu_batch_pack_cells: the blocks (IDs and 64 values) of cells[0..n_sel)
   into gids / data, DEVICE buffers on the batch's device of `capacity`
   blocks, cell after cell; counts (host, n_sel) receives each cell's block
   count and *used the total (VLGPU_ENOMEM, with *used set, when it exceeds
   capacity).

   vlgpu_batch_unpack_cells: replaces the blocks of cells[0..n_sel) with
   counts[i] blocks each, taken cell after cell from gids / data (device
   buffers on the batch's device, as vlgpu_batch_pack_cells writes them).
   The blocks are appended behind the rows in use (VLGPU_ENOMEM beyond the
   batch's capacity); a block ID outside the mesh gives VLGPU_EINVAL.

   Both work on the batch's own stream, which waits for no other stream, and
   return once it is idle.  So the caller's buffers must be complete before
   the call (synchronise the stream that received or last used them), and
   they are free to reuse when it returns. */
int vlgpu_batch_pack_cells(vlgpu_batch* b, uint32_t n_sel, const uint32_t* cells, uint32_t* counts, uint32_t* gids,
                           float* data, uint64_t capacity, uint64_t* used);
int vlgpu_batch_unpack_cells(vlgpu_batch* b, uint32_t n_sel, const uint32_t* cells, const uint32_t* counts,
                             const uint32_t* gids, const float* data);

/* Per-cell VLGPU_CELL_* bits accumulated since the last upload. */
int vlgpu_batch_status(vlgpu_batch* b, uint32_t* status);

/* ---- the hot path ------------------------------------------------------- */

/* One SLICE-3D 1D remap along `dimension` of every cell of the batch.
   Replaces map_1d (vlasovsolver/cpu_acc_map.hpp:30-32, cpu_acc_map.cpp:121-636)
   called once per cell.  intersections: 4 doubles per cell (intersection,
   di, dj, dk) in host memory, as stored in Population::intersection_*
   (spatial_cell_cpu.hpp:89-92). */
int vlgpu_map_1d(vlgpu_batch* b, const double* intersections, uint32_t dimension);

/* The same sweep issued as one launch sequence per cell (the plain per-cell
   drop-in path, vlasovsolver/cpu_acc_semilag.cpp:64-75 without OpenMP). */
int vlgpu_map_1d_per_cell(vlgpu_batch* b, const double* intersections, uint32_t dimension);

/* The same sweep for callers that must not allocate device memory.  It
   always runs the fused arithmetic with PPM (the defaults of a batch, see
   vlgpu_batch_set_exact and vlgpu_batch_set_reconstruction), whatever mode a
   batch would use.  It has no counterpart in the reference: it exists for
   host codes that reserve all of the GPU's memory for their own pool at
   start-up, and for codes that call the sweep on a latency-critical path,
   where a cudaMalloc/cudaFree would synchronise the whole device.  It
   allocates nothing: its work arrays live in one fixed device array of about
   3.3 MB inside libvlgpu.so, held by every GPU that loads the library until
   the process exits.
   Limits per call: 1..VLGPU_NOALLOC_MAX_CELLS cells, input block indices
   below VLGPU_NOALLOC_MAX_BLOCKS (offsets[n_cells] <= the limit) and at most
   VLGPU_NOALLOC_MAX_BLOCKS output blocks; larger inputs are rejected with
   VLGPU_EINVAL and a message on stderr, an output that does not fit with
   VLGPU_ENOMEM.
   Inputs: cell c owns blocks offsets[c] .. offsets[c+1]-1 (host array of
   n_cells+1) of gids_in / data_in (device memory, 64 floats per block, block
   IDs inside the mesh); intersections as for vlgpu_map_1d (host).  Outputs:
   gids_out / data_out (device memory, room for out_capacity blocks); cell c's
   blocks are cell_off[c] .. cell_off[c]+cell_count[c]-1 of them, in sweep
   order (host arrays of n_cells); status (host, may be NULL) gets each cell's
   VLGPU_CELL_* bits of this call.  data_in and data_out are 16-byte aligned.
   The output buffers must not overlap the input buffers (the sweep reads
   blocks of one cell after writing blocks of another); passing the same
   pointer for both is rejected with VLGPU_EINVAL.
   The work is issued on `stream` (a cudaStream_t of the current device, NULL
   for the default stream) and the call synchronises it before returning.
   Every call looks up the device array's address (cudaGetSymbolAddress) on
   the current device; the first call on a device also loads the library's
   kernels there, so make that first call before any stream capture begins.  Every call on a device uses the same array: calls
   that overlap on the GPU (from several host threads at once) race and must
   be serialised by the caller. */
#define VLGPU_NOALLOC_MAX_BLOCKS 65536u
#define VLGPU_NOALLOC_MAX_CELLS 1024u
int vlgpu_map_1d_noalloc(const vlgpu_mesh* mesh, const vlgpu_params* params, uint32_t n_cells,
                         const uint64_t* offsets, const uint32_t* gids_in, const float* data_in,
                         const double* intersections, uint32_t dimension, uint32_t* gids_out, float* data_out,
                         uint64_t out_capacity, uint32_t* cell_off, uint32_t* cell_count, uint32_t* status,
                         void* stream);

/* Three sweeps in map_order 0 (XYZ), 1 (YZX) or 2 (ZXY) with given
   intersections (12 doubles per cell ordered x, y, z; cpu_accelerate_cell,
   vlasovsolver/cpu_acc_semilag.cpp:92-130). */
int vlgpu_accelerate_with_intersections(vlgpu_batch* b, const double* intersections12, uint32_t map_order);

/* One acceleration step of every cell, as calculateAcceleration does for
   one population and one subcycle (vlasovsolver/vlasovmover.cpp:410-475,
   564-569): first velocity moments of the current VDF give the pivot
   (calculateMoments_V), the FP64 gyration transform and intersections are
   built per cell on the device (cpu_acc_transform.cpp:66-153,
   cpu_acc_intersections.cpp:44-450), the three sweeps run in map_order, the
   blocks are adjusted (adjustVelocityBlocks, grid.cpp:775-817, cells without
   spatial neighbours) and the moments including the pressure tensor are
   recomputed.  fields: one vlgpu_cell_fields per cell; dt: one substep length
   per cell (Population::subcycleDt); host memory.  A cell whose dt is 0 is
   not accelerated: its blocks pass through the sweeps unchanged, as the
   reference leaves cells that have finished their subcycles out of the
   accelerated cells (vlasovmover.cpp:547-556) and does no remap when dt is 0
   (vlasovmover.cpp:490-497); its block adjustment and moments still run, and
   adjusting an already adjusted cell changes nothing. */
int vlgpu_accelerate(vlgpu_batch* b, const vlgpu_cell_fields* fields, const double* dt, uint32_t map_order);

/* Only the geometry part of that step: pivot moments, FP64 transform and the
   three intersection sets of every cell (compute_cell_intersections,
   vlasovsolver/cpu_acc_intersections.cpp:44-101), readable with
   vlgpu_batch_intersections; the VDF is not changed. */
int vlgpu_compute_intersections(vlgpu_batch* b, const vlgpu_cell_fields* fields, const double* dt,
                                uint32_t map_order);

/* The same step reusing the fields and dt last passed to vlgpu_accelerate
   (no host data; suitable for stream capture). */
int vlgpu_accelerate_device(vlgpu_batch* b, uint32_t map_order);

/* The same step with every sweep issued as one launch sequence per cell: the
   plain per-cell path, kept as the drop-in baseline of the batched one. */
int vlgpu_accelerate_per_cell(vlgpu_batch* b, uint32_t map_order);

/* ---- spatial translation ------------------------------------------------ */

/* Declares the batch's cells to be a uniform periodic spatial grid of
   dims[0] x dims[1] x dims[2] cells (x fastest: cell = x + dims[0]*(y +
   dims[1]*z); dims[0]*dims[1]*dims[2] == n_cells, each dims[d] <= 128) with
   cell sizes dx[3] (m), as the reference's DX/DY/DZ cell parameters.  Adds
   translation work arrays sized from the block capacity. */
int vlgpu_batch_set_grid(vlgpu_batch* b, const uint32_t dims[3], const double dx[3]);

/* One translation sweep along `dimension` of every cell of the grid over dt
   seconds: trans_map_1d_amr (vlasovsolver/cpu_trans_map_amr.cpp:214-443,
   propagatePencil :37-150) for pencils through a uniform periodic grid.
   Block sets do not change; mass flowing into a cell that lacks the block is
   dropped, as in the reference. */
int vlgpu_translate(vlgpu_batch* b, uint32_t dimension, double dt);

/* One full Vlasov step of the grid over dt seconds, in the reference's main
   loop order: translation along z, x, y (calculateSpatialTranslation,
   vlasovsolver/vlasovmover.cpp:65-381) with the "_R" moments after it
   (calculateMoments_R, arch_moments.cpp), then one acceleration step with
   fields[] (one per cell, host) and map_order as vlgpu_accelerate does it,
   whose block adjustment consults the spatial neighbours (adjustVelocityBlocks
   with the full neighbour lists, vlasovmover.cpp:564-569).  One subcycle. */
int vlgpu_vlasov_step(vlgpu_batch* b, const vlgpu_cell_fields* fields, double dt, uint32_t map_order);

/* The same step reusing the fields last passed (no host data; the
   acceleration uses the per-cell dt last staged). */
int vlgpu_vlasov_step_device(vlgpu_batch* b, double dt, uint32_t map_order);

/* The "_R" moments computed after the last translation of a Vlasov step, in
   the layout of vlgpu_batch_moments (16 doubles per cell). */
int vlgpu_batch_moments_r(vlgpu_batch* b, double* out16);

/* Initial VDF of every cell from a Maxwellian or tri-Maxwellian
   (MaxwellianPhaseSpaceDensity / TriMaxwellianPhaseSpaceDensity,
   projects/project.h:45-73) sampled at the cell centres of the blocks around
   it (Project::setVelocitySpace, projects/project.cpp:239-260), then pruned by
   the first block adjustment (grid.cpp:289; with the spatial neighbours on a
   grid).  Replaces the cells' blocks; clears status and adjustment loss.  The
   species mass is the batch's. */
typedef struct vlgpu_maxwellian {
   double n;        /* number density, m^-3 */
   double T[3];     /* temperatures along the frame's rows, K (equal and an identity frame: isotropic) */
   double frame[9]; /* rows: the temperature axes (row-major 3x3) */
   double V[3];     /* bulk velocity, m/s */
} vlgpu_maxwellian;
int vlgpu_batch_fill_maxwellian(vlgpu_batch* b, const vlgpu_maxwellian* cells);

/* 0.5 * ("_R" + "_V") of every moment, as calculateInterpolatedVelocityMoments
   (vlasovsolver/vlasovmover.cpp:587-631) forms the moments the field solver
   reads; the "_V" set is the last one computed (vlgpu_accelerate,
   vlgpu_vlasov_step or vlgpu_batch_moments).  Grid batches. */
int vlgpu_batch_interpolated_moments(vlgpu_batch* b, double* out16);

/* Time-step limits per cell (host arrays of n_cells): r_dt = the r-space
   limit of reduce_vlasov_dt (vlasovsolver/arch_dt.cpp:34-97) from the cell's
   current blocks and the grid's cell sizes; v_dt = the v-space limit of
   updateAccelerationMaxdt (cpu_acc_transform.cpp:41-55), |gyroperiod| *
   max_rotation_deg / 360 from the fields last passed to vlgpu_accelerate or
   vlgpu_compute_intersections.  The batch must be a grid. */
int vlgpu_batch_max_dt(vlgpu_batch* b, double max_rotation_deg, double* r_dt, double* v_dt);

/* Block adjustment of every cell (SpatialCell::adjust_velocity_blocks,
   spatial_cells/spatial_cell_cpu.cpp:179-273): keeps the blocks with content and their +-blockAddWidthV velocity
   neighbours and, when the batch is a grid (vlgpu_batch_set_grid), every
   block with content in one of the cell's 26 nearest spatial neighbours
   (adjustVelocityBlocks, grid.cpp:775-817); removes the rest, adds missing
   blocks with zero data. */
int vlgpu_adjust_blocks(vlgpu_batch* b);

/* Mass removed by block adjustment per cell since the last upload
   (Population::RHOLOSSADJUST, sum f dv^3). */
int vlgpu_batch_rho_loss(vlgpu_batch* b, double* out);

/* Velocity moments of every cell's current VDF (calculateMoments_V,
   vlasovsolver/arch_moments.cpp:342-499, one population), FP64 with
   compensated sums.  The record of the last vlgpu_accelerate holds the
   post-step moments already; this call recomputes them.  out16: 16 doubles per cell: n, n*V (3), RHOM_V, V_V (3),
   RHOQ_V, P_11, P_22, P_33, P_23, P_13, P_12 (zero unless compute_second),
   sum of f. */
int vlgpu_batch_moments(vlgpu_batch* b, int compute_second, double* out16);

/* The 12 FP64 intersections per cell (x, y, z; each intersection, di, dj,
   dk) computed by the last vlgpu_accelerate. */
int vlgpu_batch_intersections(vlgpu_batch* b, double* out12);

/* The CUDA stream (cudaStream_t) all of the batch's work is issued on, for
   callers that time it with events or order their own work after it. */
int vlgpu_batch_stream(vlgpu_batch* b, void** stream);

/* Enables (1) or disables (0) CUDA-event timing of every remap launch and
   clears the accumulated time. */
int vlgpu_batch_profile(vlgpu_batch* b, int enable);

/* Counters since creation: [0] kernels launched, [1] cell-sweeps,
   [2] source blocks entering sweeps, [3] blocks written by sweeps,
   [4] remap launches, [5] profiled remap time (ns), [6] profiled remap
   launches, [7] column sets remapped.  Synchronises the stream. */
int vlgpu_batch_stats(vlgpu_batch* b, uint64_t* out8);

/* Further counters: [0] blocks that entered the first sweep of each
   acceleration step (the step's phase-space cell updates / 64). */
int vlgpu_batch_stats2(vlgpu_batch* b, uint64_t* out);

/* Selects the remap arithmetic of later sweeps.  exact = 1 evaluates every
   operation in the reference's order and rounding (cpu_acc_map.cpp:395-631),
   so VDF values and block sets are bit-identical to the reference's map_1d.
   exact = 0 (the default) keeps the reference's PPM reconstruction but
   distributes each source cell over its target cells with fused
   multiply-adds and at most three targets per source cell: block sets are
   unchanged, values stay within 1e-5 of the cell's peak per step, and mass
   is conserved as in the exact mode.  The same switch selects the
   translation's arithmetic: exact = 1 is bit-identical to trans_map_1d_amr,
   exact = 0 uses the uniform-width face, single-precision PPM and FMA. */
int vlgpu_batch_set_exact(vlgpu_batch* b, int exact);

/* Selects the acceleration reconstruction of later sweeps, the reference's
   compile-time ACC_SEMILAG_* choice (cpu_acc_map.cpp:537-548, 590-601):
   VLGPU_RECON_PLM (compute_plm_coeff, cpu_1d_plm.hpp:38-49), VLGPU_RECON_PPM
   (the default; compute_ppm_coeff, cpu_1d_ppm.hpp:35-54) or VLGPU_RECON_PQM
   (compute_pqm_coeff with h8 faces and h7 derivatives, cpu_1d_pqm.hpp:157-176,
   cpu_face_estimates.hpp:45-79, 216-275; the reference Makefile's default).
   PLM and PQM run in the fused arithmetic only (values within 1e-5 of the
   cell's peak per sweep); combining them with exact = 1 is VLGPU_EINVAL. */
#define VLGPU_RECON_PLM 1
#define VLGPU_RECON_PPM 2
#define VLGPU_RECON_PQM 4
int vlgpu_batch_set_reconstruction(vlgpu_batch* b, int order);

/* Captures n_steps (2, 4 or 6) consecutive device steps into a CUDA graph kept
   in the batch's graph slot `slot` (0..7): acceleration steps as
   vlgpu_accelerate_device does them (kind 0) or full Vlasov steps as
   vlgpu_vlasov_step_device does them with dt (kind 1, grid batches), with
   map_orders[q] for step q.  Nothing runs during the capture.  Every step
   moves the VDF between two buffer sets, so an even number of steps starts
   and ends on the same set, and the graph can be replayed any number of
   times while the batch stays in that state.  Capture after at least one
   step of the same kind (the state a step leaves), with profiling off. */
int vlgpu_batch_capture(vlgpu_batch* b, int slot, int kind, uint32_t n_steps, const uint32_t* map_orders,
                        double dt);

/* Launches the graph in `slot` on the batch's stream (asynchronously).
   VLGPU_EINVAL if the batch is not in the buffer state of the capture. */
int vlgpu_batch_replay(vlgpu_batch* b, int slot);

/* ---- launch shapes and their tuning table (no reference counterpart) ----

   The batch's persistent kernels run with a number of CTAs per SM: the
   acceleration remap (16 column sets per CTA in flight), the moments, the
   block adjustment and the translation walk.  0 means the kernel's occupancy
   maximum (the default); larger values are clamped to it.  Without a
   vlgpu_batch_set_launch call, every upload consults the tuning table written
   by vlasiator_b200/autotune.py: per device name and bucket of mean blocks
   per cell, the fastest shapes of timed steps.  The table is the file
   $VLGPU_LAUNCH_TABLE, else $XDG_CACHE_HOME/vlgpu/launch_table.tsv (~/.cache
   when XDG_CACHE_HOME is unset), lines of
   "<device>\t<lowest mean blocks>\t<remap>\t<moments>\t<adjust>\t<translate>";
   a missing file or entry means the defaults. */
typedef struct vlgpu_launch {
   uint32_t remap_ctas_per_sm;
   uint32_t moments_ctas_per_sm;
   uint32_t adjust_ctas_per_sm;
   uint32_t translate_ctas_per_sm;
} vlgpu_launch;

/* Sets the shapes (the table is then not consulted); NULL returns the batch
   to the table at its next upload. */
int vlgpu_batch_set_launch(vlgpu_batch* b, const vlgpu_launch* cfg);

/* The shapes in use (resolved CTAs per SM; translate 0 = its maximum). */
int vlgpu_batch_get_launch(vlgpu_batch* b, vlgpu_launch* cfg);

/* The table entry for a device name and mean block count (path NULL: the
   default table); VLGPU_ENOENT when there is none.  Host only. */
int vlgpu_launch_table_lookup(const char* path, const char* device, double mean_blocks, vlgpu_launch* out);

/* Synchronises the batch's stream and returns the first error seen. */
int vlgpu_batch_sync(vlgpu_batch* b);

/* ---- serving ------------------------------------------------------------ */

/* A request loop around one device-resident batch of max_cells cells: each
   request is one spatial cell's VDF to be advanced by n_steps acceleration
   steps (calculateAcceleration for one population, as vlgpu_accelerate does
   it).  Requests queue on the host, join the batch between steps while free
   cells and the block budget allow (continuous batching), keep their blocks
   on the device for their whole life and are copied back after their last
   step.  hbm_budget_bytes sizes the batch: block capacity = budget / bytes
   per block of all the batch's arrays; admission keeps the live blocks below
   60% of it.  Step s of every request uses dimension order s mod 3 and cells
   never interact, so a request's result does not depend on the requests it
   ran with.  One host thread drives a server. */
typedef struct vlgpu_server vlgpu_server;
int vlgpu_server_create(const vlgpu_mesh* mesh, const vlgpu_params* params, uint32_t max_cells,
                        uint64_t hbm_budget_bytes, int device, vlgpu_server** out);
int vlgpu_server_destroy(vlgpu_server* s);

/* Queues a request (its data are copied); *request_id identifies it. */
int vlgpu_server_submit(vlgpu_server* s, uint32_t n_blocks, const uint32_t* gids, const float* data,
                        const vlgpu_cell_fields* fields, double dt, uint32_t n_steps, uint64_t* request_id);

/* One tick: waits for the previous step, copies finished requests back,
   admits queued ones, and issues one acceleration step of all active cells
   (asynchronously).  Reports the active, queued and just-finished counts. */
int vlgpu_server_tick(vlgpu_server* s, uint32_t* n_active, uint32_t* n_pending, uint32_t* n_done);

/* The result of a finished request (blocks in ascending global-ID order, its
   VLGPU_CELL_* bits and its block-adjustment loss), then forgets it.
   VLGPU_EAGAIN while it runs; VLGPU_ENOMEM (with *n_blocks set) when
   capacity is too small. */
int vlgpu_server_result(vlgpu_server* s, uint64_t request_id, uint32_t* n_blocks, uint32_t* gids, float* data,
                        uint64_t capacity, uint32_t* status, double* rho_loss);

/* [0] ticks, [1] requests finished, [2] cell-steps run, [3] phase-space
   cell-updates (64 x blocks entering each step). */
int vlgpu_server_stats(vlgpu_server* s, uint64_t* out4);

/* The server's batch (for its stream and counters; do not destroy it). */
int vlgpu_server_batch(vlgpu_server* s, vlgpu_batch** batch);

/* Library version string. */
const char* vlgpu_version(void);

#ifdef __cplusplus
}
#endif
#endif /* VLGPU_H */
