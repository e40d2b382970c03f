// C ABI of libvlgpu.so: device-resident cell batches and the hot-path entry
// points declared in include/vlgpu.h.  The batch itself and its internal
// operations are described in batch_internal.cuh.
#include <cmath>

#include "batch_internal.cuh"

namespace vlgpu_batch_ops {

int cuda_status(cudaError_t e, const char* what) {
   if (e == cudaSuccess) return VLGPU_OK;
   std::fprintf(stderr, "vlgpu: %s: %s\n", what, cudaGetErrorString(e));
   return e == cudaErrorMemoryAllocation ? VLGPU_ENOMEM : VLGPU_ECUDA;
}

void free_batch(vlgpu_batch* b) {
   if (!b) return;
   cudaSetDevice(b->device);
   for (int p = 0; p < 2; ++p) {
      cudaFree(b->gids[p]);
      cudaFree(b->data[p]);
      cudaFree(b->slots[p]);
      cudaFree(b->adj_gids[p]);
      cudaFree(b->adj_src[p]);
      cudaFree(b->adj_slots[p]);
   }
   cudaFree(b->content);
   cudaFree(b->perm);
   cudaFree(b->sets);
   cudaFree(b->sweep_cells);
   cudaFree(b->sweep3);
   cudaFree(b->accel_in);
   cudaFree(b->moments);
   cudaFree(b->pivot);
   cudaFree(b->mom_parts);
   cudaFree(b->mom_done);
   cudaFree(b->mom_scratch);
   cudaFree(b->isect12);
   cudaFree(b->loss);
   cudaFree(b->status);
   cudaFree(b->counters);
   cudaFree(b->stats);
   cudaFree(b->rows_used);
   cudaFree(b->item_gid);
   cudaFree(b->item_pencil);
   cudaFree(b->trans_rows);
   cudaFree(b->trans_src);
   cudaFree(b->tcounters);
   cudaFree(b->neighbors);
   cudaFree(b->dt_buf);
   cudaFree(b->adj_scratch);
   cudaFree(b->wide_cells);
   cudaFree(b->halo_scratch);
   cudaFree(b->cell_order);
   if (b->h_order) cudaFreeHost(b->h_order);
   cudaFree(b->mask_recs);
   cudaFree(b->mask_pool);
   cudaFree(b->mask_top);
   cudaFree(b->moments_r);
   for (auto& g : b->graphs)
      if (g.exec) cudaGraphExecDestroy(g.exec);
   for (cudaEvent_t e : b->prof_events) cudaEventDestroy(e);
   cudaFreeHost(b->h_sweep);
   cudaFreeHost(b->h_accel);
   cudaFreeHost(b->h_slots_in);
   cudaFreeHost(b->h_slots_out);
   if (b->ev_upload) cudaEventDestroy(b->ev_upload);
   if (b->ev_order) cudaEventDestroy(b->ev_order);
   if (b->ev_slots) cudaEventDestroy(b->ev_slots);
   if (b->ev_sweep) cudaEventDestroy(b->ev_sweep);
   if (b->ev_accel) cudaEventDestroy(b->ev_accel);
   if (b->stream) cudaStreamDestroy(b->stream);
   delete b;
}

void set_direct_state(vlgpu_batch* b, int pool) {
   b->st_gids = b->gids[pool];
   b->st_src = nullptr;
   b->st_slots = b->slots[pool];
   b->cur = pool;
   b->st_list = pool;
   b->pivot_valid = false;
}

// One sweep of every cell; sweep parameters already on the device.
int sweep_device(vlgpu_batch* b, const SweepCell* sweep_cells, uint32_t dim, bool per_cell, bool first_of_step) {
   const int src = b->cur, dst = 1 - b->cur;
   const uint32_t cap = (uint32_t)b->capacity;
   const int wm = (int)b->params.wall_margin;
   const double thr = b->params.min_value;
   VL_CHECK(cudaMemsetAsync(b->counters, 0, sizeof(SweepCounters), b->stream));
   if (!per_cell) {
      VL_CHECK(launch_columnize_batch((int)dim, b->st_gids, b->st_src, b->st_slots, b->slots[dst], b->perm, b->sets,
                                      cap, cap, sweep_cells, b->status, b->counters, b->stats, b->mdev, wm,
                                      b->n_cells, first_of_step ? 1 : 0, b->wide_cells, b->cell_order,
                                      b->col_wide_grid, b->stream));
      const bool prof = b->profiling && b->prof_used + 2 <= b->prof_events.size();
      if (prof) VL_CHECK(cudaEventRecord(b->prof_events[b->prof_used], b->stream));
      VL_CHECK(launch_remap((int)dim, b->sets, b->counters, b->perm, b->data[src], b->data[dst], b->gids[dst],
                            sweep_cells, b->status, b->mdev, wm, cap, b->content, thr, b->exact, b->recon, b->remap_grid,
                            b->stream));
      if (prof) {
         VL_CHECK(cudaEventRecord(b->prof_events[b->prof_used + 1], b->stream));
         b->prof_used += 2;
      }
      b->launches += 3;
      b->remap_launches += 1;
   } else {
      // one columnize + remap launch pair per cell; set and output counters
      // keep running so the cells land in disjoint ranges
      for (uint32_t c = 0; c < b->n_cells; ++c) {
         VL_CHECK(launch_rebase_work(b->counters, b->stream));
         VL_CHECK(launch_columnize((int)dim, b->st_gids, b->st_src, b->st_slots, b->slots[dst], b->perm, b->sets,
                                   cap, cap, sweep_cells, b->status, b->counters, b->stats, b->mdev, wm, c, c + 1,
                                   first_of_step ? 1 : 0, b->stream));
         VL_CHECK(launch_remap((int)dim, b->sets, b->counters, b->perm, b->data[src], b->data[dst], b->gids[dst],
                               sweep_cells, b->status, b->mdev, wm, cap, b->content, thr, b->exact, b->recon, b->sm_count,
                               b->stream));
         b->launches += 3;
         b->remap_launches += 1;
      }
   }
   VL_CHECK(cudaMemcpyAsync(b->rows_used + dst, &b->counters->dst_top, sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                            b->stream));
   set_direct_state(b, dst);
   b->content_valid = true;
   return VLGPU_OK;
}

// One sweep with host-given intersections (4 doubles per cell at `stride`).
int run_sweep(vlgpu_batch* b, const double* intersections, size_t stride, uint32_t dim, bool per_cell) {
   VL_CHECK(cudaEventSynchronize(b->ev_sweep));  // the previous copy out of h_sweep has been read
   for (uint32_t c = 0; c < b->n_cells; ++c)
      b->h_sweep[c] = make_sweep_cell(intersections + stride * c, dim, b->params.min_value);
   VL_CHECK(cudaMemcpyAsync(b->sweep_cells, b->h_sweep, sizeof(SweepCell) * b->n_cells, cudaMemcpyHostToDevice,
                            b->stream));
   VL_CHECK(cudaEventRecord(b->ev_sweep, b->stream));
   return sweep_device(b, b->sweep_cells, dim, per_cell, false);
}

int moments_device(vlgpu_batch* b, bool second, double* record, const double* shift) {
   b->launches += 1;
   VL_CHECK(launch_moments(b->st_gids, b->st_src, b->data[b->cur], b->st_slots, record ? record : b->moments, shift,
                           b->mdev, b->vmin_d, b->bs_d, b->dv_d, b->params.mass, b->params.charge, second,
                           b->n_cells, b->mom_parts, b->mom_done, b->mom_grid, b->stream));
   return VLGPU_OK;
}

// First and second moments of the current VDF in one read: the second about
// the bulk velocity in the pivot record (any earlier VDF's, or zero), which
// then receives this VDF's first moments; the full record goes to `record`.
int moments_both_device(vlgpu_batch* b, double* record) {
   b->launches += 1;
   VL_CHECK(launch_moments_both(b->st_gids, b->st_src, b->data[b->cur], b->st_slots, b->pivot, record, b->mdev,
                                b->vmin_d, b->bs_d, b->dv_d, b->params.mass, b->params.charge, b->n_cells,
                                b->mom_parts, b->mom_done, b->mom_grid, b->stream));
   b->pivot_valid = true;
   return VLGPU_OK;
}

// Block adjustment of every cell; with `record`, the same pass also gives the
// adjusted VDF's "_V" moments (MOM_BOTH: first moments about 0, pressure
// about the pivot's bulk velocity) into `record`, and with write_pivot its
// first moments become the next acceleration's pivot.
int adjust_device(vlgpu_batch* b, double* record, bool write_pivot) {
   const int a = b->adj_next;
   b->adj_next = 1 - a;
   VL_CHECK(cudaMemsetAsync(b->counters, 0, sizeof(SweepCounters), b->stream));
   const double dv3 = b->dv_d[0] * b->dv_d[1] * b->dv_d[2];
   MomentFrame frame{};
   for (int d = 0; d < 3; ++d) {
      frame.vmin[d] = b->vmin_d[d];
      frame.bs[d] = b->bs_d[d];
      frame.dv[d] = b->dv_d[d];
   }
   frame.mass = b->params.mass;
   frame.charge = b->params.charge;
   VL_CHECK(launch_adjust(b->st_gids, b->st_src, b->st_slots, b->content_valid ? b->content : nullptr,
                          b->data[b->cur], b->neighbors, b->adj_gids[a], b->adj_src[a], b->adj_slots[a], b->loss,
                          b->status,
                          b->counters, (uint32_t)b->capacity, b->mdev, b->params.min_value,
                          (int)b->params.add_width_v, dv3, b->n_cells, b->adj_scratch, b->adj_grid,
                          b->cell_order, b->mask_recs, b->mask_pool, b->mask_top, b->mask_cap, record, b->pivot,
                          write_pivot ? 1 : 0, frame, b->stream));
   b->launches += (b->neighbors && b->mask_recs) ? 2 : 1;  // content masks first on a grid
   VL_CHECK(cudaMemcpyAsync(b->rows_used + 2 + a, &b->counters->dst_top, sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                            b->stream));
   b->st_gids = b->adj_gids[a];
   b->st_src = b->adj_src[a];
   b->st_slots = b->adj_slots[a];
   b->st_list = 2 + a;
   b->content_valid = false;
   b->pivot_valid = record && write_pivot;
   return VLGPU_OK;
}

// Copies an indirect state's values into the other pool in list order.
int materialize(vlgpu_batch* b) {
   if (!b->st_src) return VLGPU_OK;
   std::vector<CellSlot> slots(b->n_cells);
   VL_CHECK(cudaMemcpyAsync(slots.data(), b->st_slots, sizeof(CellSlot) * b->n_cells, cudaMemcpyDeviceToHost,
                            b->stream));
   VL_CHECK(cudaStreamSynchronize(b->stream));
   uint64_t hi = 0;
   for (const CellSlot& s : slots) hi = std::max<uint64_t>(hi, (uint64_t)s.off + s.count);
   const int dst = 1 - b->cur;
   VL_CHECK(launch_materialize(b->st_src, b->data[b->cur], b->data[dst], hi, b->stream));
   b->launches += 1;
   VL_CHECK(cudaMemcpyAsync(b->rows_used + dst, b->rows_used + b->st_list, sizeof(uint32_t),
                            cudaMemcpyDeviceToDevice, b->stream));
   b->st_src = nullptr;
   b->cur = dst;
   b->pivot_valid = false;
   return VLGPU_OK;
}

// The same without a host round trip: the row count stays on the device.
int materialize_async(vlgpu_batch* b) {
   if (!b->st_src) return VLGPU_OK;
   const int dst = 1 - b->cur;
   VL_CHECK(launch_materialize_rows(b->st_src, b->data[b->cur], b->data[dst], b->rows_used + b->st_list,
                                    b->sm_count * 8, b->stream));
   b->launches += 1;
   VL_CHECK(cudaMemcpyAsync(b->rows_used + dst, b->rows_used + b->st_list, sizeof(uint32_t),
                            cudaMemcpyDeviceToDevice, b->stream));
   b->st_src = nullptr;
   b->cur = dst;
   return VLGPU_OK;
}

// Pivot moments and the per-cell FP64 geometry of one acceleration step.
int geometry_device(vlgpu_batch* b, uint32_t map_order) {
   // pivot velocity from the current VDF (calculateMoments_V, vlasovmover.cpp:420),
   // unless the moments that ended the previous step or the Vlasov step's "_R"
   // moments already wrote it for this VDF
   if (!b->pivot_valid) {
      const int st = moments_device(b, false, b->pivot);
      if (st != VLGPU_OK) return st;
      b->pivot_valid = true;
   }
   b->launches += 1;
   VL_CHECK(launch_geometry(b->accel_in, b->pivot, b->isect12, b->sweep3, b->n_cells, b->params.charge,
                            b->params.mass, b->params.hall_minimum_rhoq, (int)b->params.ohm_gradpe, MU_0, b->vmin_d,
                            b->dv_d, map_order, (float)b->params.min_value, b->stream));
   return VLGPU_OK;
}

int accelerate_device(vlgpu_batch* b, uint32_t map_order, bool per_cell, bool next_pivot) {
   int st = geometry_device(b, map_order);
   if (st != VLGPU_OK) return st;
   static const uint32_t orders[3][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}};
   for (int s = 0; s < 3; ++s) {
      const uint32_t d = orders[map_order][s];
      st = sweep_device(b, b->sweep3 + (size_t)d * b->n_cells, d, per_cell, s == 0);
      if (st != VLGPU_OK) return st;
   }
   // final block adjustment and moments (vlasovmover.cpp:564-569), in one
   // pass: the "_V" moments of the adjusted VDF, and with next_pivot its first
   // moments as the next step's pivot
   return adjust_device(b, b->moments, next_pivot);
}

// One translation sweep of the whole grid along `dim` (trans_map_1d_amr):
// out of place into the other pool, same block lists.
int translate_device(vlgpu_batch* b, uint32_t dim, double dt) {
   const int d = 1 - b->cur;
   const uint32_t N = b->grid_dims[dim];
   VL_CHECK(cudaMemsetAsync(b->tcounters, 0, sizeof(TransCounters), b->stream));
   VL_CHECK(launch_pencil_union(b->st_gids, b->st_slots, (int)dim, b->grid_dims[0], b->grid_dims[1],
                                b->grid_dims[2], b->mdev, b->item_gid, b->item_pencil, b->trans_rows,
                                b->trans_src, b->st_src, (uint32_t)b->capacity, b->row_cap, b->tcounters, b->status,
                                b->stream));
   int per_sm = trans_blocks_per_sm(N, b->exact);
   if (b->cps[3] > 0 && (int)b->cps[3] < per_sm) per_sm = (int)b->cps[3];
   const int grid = b->sm_count * per_sm;
   VL_CHECK(launch_trans_remap((int)dim, N, b->item_gid, b->item_pencil, b->trans_rows, b->trans_src, b->tcounters,
                               (uint32_t)b->capacity, b->row_cap, b->st_src, b->data[b->cur], b->data[d], b->gids[d],
                               b->mdev, (float)dt, (float)b->grid_dx[dim], (float)b->params.min_value, b->exact, grid,
                               b->stream));
   VL_CHECK(cudaMemcpyAsync(b->slots[d], b->st_slots, sizeof(CellSlot) * b->n_cells, cudaMemcpyDeviceToDevice,
                            b->stream));
   VL_CHECK(cudaMemcpyAsync(b->rows_used + d, b->rows_used + b->st_list, sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                            b->stream));
   b->launches += 2;
   set_direct_state(b, d);
   b->content_valid = false;
   return VLGPU_OK;
}

// One full Vlasov step of a grid: translation z, x, y and the "_R" moments
// (calculateSpatialTranslation, vlasovmover.cpp:65-381), then one acceleration
// step with its final adjustment and "_V" moments (calculateAcceleration,
// vlasovmover.cpp:410-581), as the reference's main loop orders them.
int vlasov_step_device(vlgpu_batch* b, double dt, uint32_t map_order) {
   static const uint32_t trans_order[3] = {2, 0, 1};
   for (int s = 0; s < 3; ++s) {
      const int st = translate_device(b, trans_order[s], dt);
      if (st != VLGPU_OK) return st;
   }
   // "_R" moments; their first pass is also the acceleration's pivot record
   const int st = moments_both_device(b, b->moments_r);
   if (st != VLGPU_OK) return st;
   b->pivot_valid = true;
   // the next step starts with a translation, so its pivot is found anew
   return accelerate_device(b, map_order, false, false);
}

int stage_fields(vlgpu_batch* b, const vlgpu_cell_fields* fields, const double* dt) {
   VL_CHECK(cudaEventSynchronize(b->ev_accel));  // the previous copy out of h_accel has been read
   for (uint32_t c = 0; c < b->n_cells; ++c) {
      CellAccelInputs& a = b->h_accel[c];
      for (int r = 0; r < 3; ++r) {
         a.B[r] = fields[c].B[r];
         a.curl[r] = fields[c].curl[r];
         a.egradpe[r] = fields[c].egradpe[r];
      }
      a.dt = dt[c];
   }
   VL_CHECK(cudaMemcpyAsync(b->accel_in, b->h_accel, sizeof(CellAccelInputs) * b->n_cells, cudaMemcpyHostToDevice,
                            b->stream));
   VL_CHECK(cudaEventRecord(b->ev_accel, b->stream));
   return VLGPU_OK;
}

}  // namespace vlgpu_batch_ops

using namespace vlgpu_batch_ops;

extern "C" {

const char* vlgpu_version(void) { return "vlgpu 0.2 (sm_100a)"; }

int vlgpu_batch_create(const vlgpu_mesh* mesh, const vlgpu_params* params, uint32_t n_cells, uint64_t block_capacity,
                       int device, vlgpu_batch** out) {
   if (!mesh || !params || !out || n_cells == 0 || block_capacity == 0 || block_capacity >= 0xffffffffull)
      return VLGPU_EINVAL;
   for (int d = 0; d < 3; ++d)
      if (mesh->len[d] == 0 || mesh->len[d] > (uint32_t)MAX_LEN || !(mesh->vmax[d] > mesh->vmin[d]))
         return VLGPU_EINVAL;
   if (params->add_width_v > 31 || !(params->min_value > 0.0) || !(params->mass > 0.0)) return VLGPU_EINVAL;
   int ndev = 0;
   if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return VLGPU_ENODEV;
   if (device < 0 || device >= ndev) return VLGPU_EINVAL;
   vlgpu_batch* b = new vlgpu_batch();
   b->device = device;
   b->mesh = *mesh;
   b->params = *params;
   b->n_cells = n_cells;
   b->capacity = block_capacity;
   for (int d = 0; d < 3; ++d) {
      b->mdev.len[d] = mesh->len[d];
      b->vmin_d[d] = mesh->vmin[d];
      b->bs_d[d] = (mesh->vmax[d] - mesh->vmin[d]) / mesh->len[d];
      b->dv_d[d] = b->bs_d[d] / WID;
      b->mdev.dv[d] = (float)b->dv_d[d];
      b->mdev.vmin[d] = (float)mesh->vmin[d];
   }
   set_block_reciprocals(b->mdev);
   auto fail = [&](cudaError_t e, const char* what) {
      int s = cuda_status(e, what);
      free_batch(b);
      return s;
   };
   cudaError_t e = cudaSetDevice(device);
   if (e != cudaSuccess) return fail(e, "cudaSetDevice");
   if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "stream");
   cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, device);
   {
      cudaDeviceProp prop;
      if (cudaGetDeviceProperties(&prop, device) == cudaSuccess)
         std::snprintf(b->device_name, sizeof b->device_name, "%s", prop.name);
   }
   b->cps_max[0] = remap_blocks_per_sm();
   b->cps_max[1] = moments_blocks_per_sm();
   b->cps_max[2] = adjust_blocks_per_sm();
   b->col_wide_grid = b->sm_count * columnize_wide_blocks_per_sm(b->mdev);
   apply_launch(b);
   const uint64_t cap = block_capacity;
   for (int p = 0; p < 2; ++p) {
      if ((e = cudaMalloc(&b->gids[p], sizeof(uint32_t) * cap)) != cudaSuccess) return fail(e, "gids");
      if ((e = cudaMalloc(&b->data[p], sizeof(float) * WID3 * cap)) != cudaSuccess) return fail(e, "data");
      if ((e = cudaMalloc(&b->slots[p], sizeof(CellSlot) * n_cells)) != cudaSuccess) return fail(e, "slots");
      if ((e = cudaMemset(b->slots[p], 0, sizeof(CellSlot) * n_cells)) != cudaSuccess) return fail(e, "slots");
      if ((e = cudaMalloc(&b->adj_gids[p], sizeof(uint32_t) * cap)) != cudaSuccess) return fail(e, "adj");
      if ((e = cudaMalloc(&b->adj_src[p], sizeof(uint32_t) * cap)) != cudaSuccess) return fail(e, "adj");
      if ((e = cudaMalloc(&b->adj_slots[p], sizeof(CellSlot) * n_cells)) != cudaSuccess) return fail(e, "adj");
   }
   if ((e = cudaMalloc(&b->content, cap)) != cudaSuccess) return fail(e, "content");
   if ((e = cudaMalloc(&b->perm, sizeof(uint32_t) * cap)) != cudaSuccess) return fail(e, "perm");
   if ((e = cudaMalloc(&b->sets, sizeof(ColumnSet) * cap)) != cudaSuccess) return fail(e, "sets");
   if ((e = cudaMalloc(&b->sweep_cells, sizeof(SweepCell) * n_cells)) != cudaSuccess) return fail(e, "sweep");
   if ((e = cudaMalloc(&b->sweep3, sizeof(SweepCell) * 3 * n_cells)) != cudaSuccess) return fail(e, "sweep3");
   if ((e = cudaMalloc(&b->accel_in, sizeof(CellAccelInputs) * n_cells)) != cudaSuccess) return fail(e, "accel");
   if ((e = cudaMemset(b->accel_in, 0, sizeof(CellAccelInputs) * n_cells)) != cudaSuccess) return fail(e, "accel");
   if ((e = cudaMalloc(&b->moments, sizeof(double) * MOM_COUNT * n_cells)) != cudaSuccess) return fail(e, "mom");
   if ((e = cudaMemset(b->moments, 0, sizeof(double) * MOM_COUNT * n_cells)) != cudaSuccess) return fail(e, "mom");
   if ((e = cudaMalloc(&b->pivot, sizeof(double) * MOM_COUNT * n_cells)) != cudaSuccess) return fail(e, "mom");
   if ((e = cudaMalloc(&b->mom_scratch, sizeof(double) * MOM_COUNT * n_cells)) != cudaSuccess) return fail(e, "mom");
   if ((e = cudaMemset(b->pivot, 0, sizeof(double) * MOM_COUNT * n_cells)) != cudaSuccess) return fail(e, "mom");
   if ((e = cudaMalloc(&b->mom_parts, sizeof(double) * MOM_SUMS_PER_PART * MOM_PARTS_PER_CELL * n_cells)) !=
       cudaSuccess)
      return fail(e, "mom");
   if ((e = cudaMalloc(&b->mom_done, sizeof(uint32_t) * n_cells)) != cudaSuccess) return fail(e, "mom");
   if ((e = cudaMemset(b->mom_done, 0, sizeof(uint32_t) * n_cells)) != cudaSuccess) return fail(e, "mom");
   if ((e = cudaMalloc(&b->isect12, sizeof(double) * 12 * n_cells)) != cudaSuccess) return fail(e, "isect");
   if ((e = cudaMemset(b->isect12, 0, sizeof(double) * 12 * n_cells)) != cudaSuccess) return fail(e, "isect");
   if ((e = cudaMalloc(&b->loss, sizeof(double) * n_cells)) != cudaSuccess) return fail(e, "loss");
   if ((e = cudaMemset(b->loss, 0, sizeof(double) * n_cells)) != cudaSuccess) return fail(e, "loss");
   if ((e = cudaMalloc(&b->status, sizeof(uint32_t) * n_cells)) != cudaSuccess) return fail(e, "status");
   if ((e = cudaMemset(b->status, 0, sizeof(uint32_t) * n_cells)) != cudaSuccess) return fail(e, "status");
   if ((e = cudaMalloc(&b->counters, sizeof(SweepCounters))) != cudaSuccess) return fail(e, "counters");
   // no sweep has run: vlgpu_batch_sync reads the overflow flag from here
   if ((e = cudaMemset(b->counters, 0, sizeof(SweepCounters))) != cudaSuccess) return fail(e, "counters");
   if ((e = cudaMalloc(&b->stats, sizeof(BatchStats))) != cudaSuccess) return fail(e, "stats");
   if ((e = cudaMalloc(&b->rows_used, sizeof(uint32_t) * 4)) != cudaSuccess) return fail(e, "rows");
   if ((e = cudaMalloc(&b->adj_scratch, sizeof(uint32_t) * adjust_scratch_words(b->mdev) *
                                            (size_t)std::min<uint32_t>((uint32_t)b->adj_grid, n_cells))) !=
       cudaSuccess)
      return fail(e, "adjust scratch");
   if ((e = cudaMalloc(&b->wide_cells, sizeof(uint32_t) * n_cells)) != cudaSuccess) return fail(e, "wide");
   if ((e = cudaMalloc(&b->cell_order, sizeof(uint32_t) * n_cells)) != cudaSuccess) return fail(e, "order");
   if ((e = cudaMallocHost(&b->h_order, sizeof(uint32_t) * n_cells)) != cudaSuccess) return fail(e, "order");
   for (uint32_t c = 0; c < n_cells; ++c) b->h_order[c] = c;
   if ((e = cudaMemcpy(b->cell_order, b->h_order, sizeof(uint32_t) * n_cells, cudaMemcpyHostToDevice)) !=
       cudaSuccess)
      return fail(e, "order");
   if ((e = cudaMemset(b->rows_used, 0, sizeof(uint32_t) * 4)) != cudaSuccess) return fail(e, "rows");
   if ((e = cudaMemset(b->stats, 0, sizeof(BatchStats))) != cudaSuccess) return fail(e, "stats");
   if ((e = cudaMallocHost(&b->h_sweep, sizeof(SweepCell) * n_cells)) != cudaSuccess) return fail(e, "pinned");
   if ((e = cudaMallocHost(&b->h_accel, sizeof(CellAccelInputs) * n_cells)) != cudaSuccess) return fail(e, "pinned");
   if ((e = cudaEventCreateWithFlags(&b->ev_sweep, cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
   if ((e = cudaEventCreateWithFlags(&b->ev_accel, cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
   if ((e = cudaMallocHost(&b->h_slots_in, sizeof(CellSlot) * (n_cells + 1))) != cudaSuccess) return fail(e, "pinned");
   if ((e = cudaHostAlloc(&b->h_slots_out, sizeof(CellSlot) * n_cells, cudaHostAllocMapped)) != cudaSuccess)
      return fail(e, "pinned");
   if ((e = cudaHostGetDevicePointer(&b->d_slots_out, b->h_slots_out, 0)) != cudaSuccess) return fail(e, "pinned");
   if ((e = cudaEventCreateWithFlags(&b->ev_upload, cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
   if ((e = cudaEventCreateWithFlags(&b->ev_order, cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
   if ((e = cudaEventCreateWithFlags(&b->ev_slots, cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
   set_direct_state(b, 0);
   *out = b;
   return VLGPU_OK;
}

int vlgpu_batch_destroy(vlgpu_batch* b) {
   if (!b) return VLGPU_EINVAL;
   if (b->stream) cudaStreamSynchronize(b->stream);
   free_batch(b);
   return VLGPU_OK;
}

// The cells by decreasing block count, for the warp-per-cell kernels (the
// longest cells start first).  Waits for the previous copy of the staging
// buffer, then copies it on the batch's stream.
static cudaError_t upload_cell_order(vlgpu_batch* b, const uint64_t* offsets) {
   cudaError_t e = cudaEventSynchronize(b->ev_order);
   if (e != cudaSuccess) return e;
   uint32_t* o = b->h_order;
   for (uint32_t c = 0; c < b->n_cells; ++c) o[c] = c;
   std::stable_sort(o, o + b->n_cells, [&](uint32_t a, uint32_t c) {
      return offsets[a + 1] - offsets[a] > offsets[c + 1] - offsets[c];
   });
   e = cudaMemcpyAsync(b->cell_order, o, sizeof(uint32_t) * b->n_cells, cudaMemcpyHostToDevice, b->stream);
   if (e != cudaSuccess) return e;
   return cudaEventRecord(b->ev_order, b->stream);
}

int vlgpu_batch_upload(vlgpu_batch* b, const uint64_t* offsets, const uint32_t* gids, const float* data) {
   if (!b || !offsets) return VLGPU_EINVAL;
   const uint64_t total = offsets[b->n_cells];
   if (total > b->capacity) return VLGPU_ENOMEM;
   if (total > 0 && (!gids || !data)) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   std::vector<CellSlot> slots(b->n_cells);
   for (uint32_t c = 0; c < b->n_cells; ++c) {
      if (offsets[c + 1] < offsets[c]) return VLGPU_EINVAL;
      slots[c].off = (uint32_t)offsets[c];
      slots[c].count = (uint32_t)(offsets[c + 1] - offsets[c]);
   }
   const uint32_t maxgid = b->mesh.len[0] * b->mesh.len[1] * b->mesh.len[2];
   for (uint64_t q = 0; q < total; ++q)
      if (gids[q] >= maxgid) return VLGPU_EINVAL;
   VL_CHECK(cudaStreamSynchronize(b->stream));
   if (total > 0) {
      VL_CHECK(cudaMemcpyAsync(b->gids[0], gids, sizeof(uint32_t) * total, cudaMemcpyHostToDevice, b->stream));
      VL_CHECK(cudaMemcpyAsync(b->data[0], data, sizeof(float) * WID3 * total, cudaMemcpyHostToDevice, b->stream));
   }
   VL_CHECK(cudaMemcpyAsync(b->slots[0], slots.data(), sizeof(CellSlot) * b->n_cells, cudaMemcpyHostToDevice,
                            b->stream));
   VL_CHECK(upload_cell_order(b, offsets));
   VL_CHECK(cudaMemsetAsync(b->status, 0, sizeof(uint32_t) * b->n_cells, b->stream));
   VL_CHECK(cudaMemsetAsync(b->loss, 0, sizeof(double) * b->n_cells, b->stream));
   VL_CHECK(cudaStreamSynchronize(b->stream));
   {
      const uint32_t used = (uint32_t)total;
      VL_CHECK(cudaMemcpy(b->rows_used, &used, sizeof(uint32_t), cudaMemcpyHostToDevice));
   }
   set_direct_state(b, 0);
   b->content_valid = false;
   consult_launch_table(b, (double)total / b->n_cells);
   return VLGPU_OK;
}

int vlgpu_batch_upload_async(vlgpu_batch* b, const uint64_t* offsets, const uint32_t* gids, const float* data) {
   if (!b || !offsets) return VLGPU_EINVAL;
   const uint64_t total = offsets[b->n_cells];
   if (total > b->capacity) return VLGPU_ENOMEM;
   if (total > 0 && (!gids || !data)) return VLGPU_EINVAL;
   for (uint32_t c = 0; c < b->n_cells; ++c)
      if (offsets[c + 1] < offsets[c]) return VLGPU_EINVAL;
   const uint32_t maxgid = b->mesh.len[0] * b->mesh.len[1] * b->mesh.len[2];
   for (uint64_t q = 0; q < total; ++q)
      if (gids[q] >= maxgid) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   VL_CHECK(cudaEventSynchronize(b->ev_upload));  // the previous upload has read the staging buffer
   CellSlot* hs = b->h_slots_in;
   for (uint32_t c = 0; c < b->n_cells; ++c) hs[c] = CellSlot{(uint32_t)offsets[c], (uint32_t)(offsets[c + 1] - offsets[c])};
   hs[b->n_cells] = CellSlot{(uint32_t)total, 0u};
   if (total > 0) {
      VL_CHECK(cudaMemcpyAsync(b->gids[0], gids, sizeof(uint32_t) * total, cudaMemcpyHostToDevice, b->stream));
      VL_CHECK(cudaMemcpyAsync(b->data[0], data, sizeof(float) * WID3 * total, cudaMemcpyHostToDevice, b->stream));
   }
   VL_CHECK(cudaMemcpyAsync(b->slots[0], hs, sizeof(CellSlot) * b->n_cells, cudaMemcpyHostToDevice, b->stream));
   VL_CHECK(upload_cell_order(b, offsets));
   VL_CHECK(cudaMemcpyAsync(b->rows_used, &hs[b->n_cells].off, sizeof(uint32_t), cudaMemcpyHostToDevice, b->stream));
   VL_CHECK(cudaMemsetAsync(b->status, 0, sizeof(uint32_t) * b->n_cells, b->stream));
   VL_CHECK(cudaMemsetAsync(b->loss, 0, sizeof(double) * b->n_cells, b->stream));
   VL_CHECK(cudaEventRecord(b->ev_upload, b->stream));
   set_direct_state(b, 0);
   b->content_valid = false;
   consult_launch_table(b, (double)hs[b->n_cells].off / b->n_cells);
   return VLGPU_OK;
}

int vlgpu_batch_download_begin(vlgpu_batch* b) {
   if (!b) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   const int st = materialize_async(b);
   if (st != VLGPU_OK) return st;
   VL_CHECK(launch_slots_to_host(b->st_slots, b->d_slots_out, b->n_cells, b->stream));
   b->launches += 1;
   VL_CHECK(cudaEventRecord(b->ev_slots, b->stream));
   return VLGPU_OK;
}

int vlgpu_batch_download_end(vlgpu_batch* b, uint32_t* cell_off, uint32_t* cell_count, uint32_t* gids, float* data,
                             uint64_t capacity, uint64_t* used) {
   if (!b || !cell_off || !cell_count || !used) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   VL_CHECK(cudaEventSynchronize(b->ev_slots));
   uint64_t hi = 0;
   for (uint32_t c = 0; c < b->n_cells; ++c) {
      cell_off[c] = b->h_slots_out[c].off;
      cell_count[c] = b->h_slots_out[c].count;
      hi = std::max<uint64_t>(hi, (uint64_t)cell_off[c] + cell_count[c]);
   }
   *used = hi;
   if (hi > capacity) return VLGPU_ENOMEM;
   if (hi > 0 && (!gids || !data)) return VLGPU_EINVAL;
   if (hi > 0) {
      VL_CHECK(cudaMemcpyAsync(gids, b->st_gids, sizeof(uint32_t) * hi, cudaMemcpyDeviceToHost, b->stream));
      VL_CHECK(cudaMemcpyAsync(data, b->data[b->cur], sizeof(float) * WID3 * hi, cudaMemcpyDeviceToHost, b->stream));
   }
   return VLGPU_OK;
}

int vlgpu_batch_block_counts(vlgpu_batch* b, uint32_t* counts) {
   if (!b || !counts) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   std::vector<CellSlot> slots(b->n_cells);
   VL_CHECK(cudaMemcpyAsync(slots.data(), b->st_slots, sizeof(CellSlot) * b->n_cells, cudaMemcpyDeviceToHost,
                            b->stream));
   VL_CHECK(cudaStreamSynchronize(b->stream));
   for (uint32_t c = 0; c < b->n_cells; ++c) counts[c] = slots[c].count;
   return VLGPU_OK;
}

int vlgpu_batch_status(vlgpu_batch* b, uint32_t* status) {
   if (!b || !status) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   VL_CHECK(cudaMemcpyAsync(status, b->status, sizeof(uint32_t) * b->n_cells, cudaMemcpyDeviceToHost, b->stream));
   VL_CHECK(cudaStreamSynchronize(b->stream));
   return VLGPU_OK;
}

int vlgpu_batch_download_raw(vlgpu_batch* b, uint32_t* cell_off, uint32_t* cell_count, uint32_t* gids, float* data,
                             uint64_t capacity, uint64_t* used) {
   if (!b || !cell_off || !cell_count || !used) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   int st = materialize(b);
   if (st != VLGPU_OK) return st;
   std::vector<CellSlot> slots(b->n_cells);
   VL_CHECK(cudaMemcpyAsync(slots.data(), b->st_slots, sizeof(CellSlot) * b->n_cells, cudaMemcpyDeviceToHost,
                            b->stream));
   VL_CHECK(cudaStreamSynchronize(b->stream));
   uint64_t hi = 0;
   for (uint32_t c = 0; c < b->n_cells; ++c) {
      cell_off[c] = slots[c].off;
      cell_count[c] = slots[c].count;
      hi = std::max<uint64_t>(hi, (uint64_t)slots[c].off + slots[c].count);
   }
   *used = hi;
   if (hi > capacity) return VLGPU_ENOMEM;
   if (hi > 0 && (!gids || !data)) return VLGPU_EINVAL;
   VL_CHECK(cudaMemcpyAsync(gids, b->st_gids, sizeof(uint32_t) * hi, cudaMemcpyDeviceToHost, b->stream));
   VL_CHECK(cudaMemcpyAsync(data, b->data[b->cur], sizeof(float) * WID3 * hi, cudaMemcpyDeviceToHost, b->stream));
   VL_CHECK(cudaStreamSynchronize(b->stream));
   return VLGPU_OK;
}

int vlgpu_batch_download(vlgpu_batch* b, uint64_t* offsets, uint32_t* gids, float* data, uint64_t capacity) {
   if (!b || !offsets) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   int st = materialize(b);
   if (st != VLGPU_OK) return st;
   std::vector<CellSlot> slots(b->n_cells);
   VL_CHECK(cudaMemcpyAsync(slots.data(), b->st_slots, sizeof(CellSlot) * b->n_cells, cudaMemcpyDeviceToHost,
                            b->stream));
   VL_CHECK(cudaStreamSynchronize(b->stream));
   uint64_t total = 0, hi = 0;
   for (uint32_t c = 0; c < b->n_cells; ++c) {
      total += slots[c].count;
      hi = std::max<uint64_t>(hi, (uint64_t)slots[c].off + slots[c].count);
   }
   offsets[0] = 0;
   for (uint32_t c = 0; c < b->n_cells; ++c) offsets[c + 1] = offsets[c] + slots[c].count;
   if (total > capacity) return VLGPU_ENOMEM;
   if (total > 0 && (!gids || !data)) return VLGPU_EINVAL;
   std::vector<uint32_t> g(hi);
   std::vector<float> d((size_t)hi * WID3);
   VL_CHECK(cudaMemcpyAsync(g.data(), b->st_gids, sizeof(uint32_t) * hi, cudaMemcpyDeviceToHost, b->stream));
   VL_CHECK(cudaMemcpyAsync(d.data(), b->data[b->cur], sizeof(float) * WID3 * hi, cudaMemcpyDeviceToHost, b->stream));
   VL_CHECK(cudaStreamSynchronize(b->stream));
   std::vector<uint32_t> order;
   for (uint32_t c = 0; c < b->n_cells; ++c) {
      const CellSlot s = slots[c];
      order.resize(s.count);
      std::iota(order.begin(), order.end(), 0u);
      std::sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return g[s.off + x] < g[s.off + y]; });
      for (uint32_t q = 0; q < s.count; ++q) {
         gids[offsets[c] + q] = g[s.off + order[q]];
         std::memcpy(data + (offsets[c] + q) * WID3, d.data() + (size_t)(s.off + order[q]) * WID3,
                     sizeof(float) * WID3);
      }
   }
   return VLGPU_OK;
}

int vlgpu_map_1d(vlgpu_batch* b, const double* intersections, uint32_t dimension) {
   if (!b || !intersections || dimension > 2) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   return run_sweep(b, intersections, 4, dimension, false);
}

int vlgpu_map_1d_per_cell(vlgpu_batch* b, const double* intersections, uint32_t dimension) {
   if (!b || !intersections || dimension > 2) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   return run_sweep(b, intersections, 4, dimension, true);
}

int vlgpu_accelerate_with_intersections(vlgpu_batch* b, const double* intersections12, uint32_t map_order) {
   if (!b || !intersections12 || map_order > 2) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   static const uint32_t orders[3][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}};
   for (int s = 0; s < 3; ++s) {
      const uint32_t d = orders[map_order][s];
      int st = run_sweep(b, intersections12 + 4 * d, 12, d, false);
      if (st != VLGPU_OK) return st;
   }
   return VLGPU_OK;
}

int vlgpu_accelerate(vlgpu_batch* b, const vlgpu_cell_fields* fields, const double* dt, uint32_t map_order) {
   if (!b || !fields || !dt || map_order > 2) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   int st = stage_fields(b, fields, dt);
   if (st != VLGPU_OK) return st;
   return accelerate_device(b, map_order, false);
}

int vlgpu_compute_intersections(vlgpu_batch* b, const vlgpu_cell_fields* fields, const double* dt,
                                uint32_t map_order) {
   if (!b || !fields || !dt || map_order > 2) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   int st = stage_fields(b, fields, dt);
   if (st != VLGPU_OK) return st;
   return geometry_device(b, map_order);
}

int vlgpu_accelerate_device(vlgpu_batch* b, uint32_t map_order) {
   if (!b || map_order > 2) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   return accelerate_device(b, map_order, false);
}

int vlgpu_accelerate_per_cell(vlgpu_batch* b, uint32_t map_order) {
   if (!b || map_order > 2) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   return accelerate_device(b, map_order, true);
}

int vlgpu_adjust_blocks(vlgpu_batch* b) {
   if (!b) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   return adjust_device(b);
}

int vlgpu_batch_rho_loss(vlgpu_batch* b, double* out) {
   if (!b || !out) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   VL_CHECK(cudaMemcpyAsync(out, b->loss, sizeof(double) * b->n_cells, cudaMemcpyDeviceToHost, b->stream));
   VL_CHECK(cudaStreamSynchronize(b->stream));
   return VLGPU_OK;
}

int vlgpu_batch_moments(vlgpu_batch* b, int compute_second, double* out16) {
   if (!b || !out16) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   const int st = compute_second ? moments_both_device(b, b->moments) : moments_device(b, false);
   if (st != VLGPU_OK) return st;
   VL_CHECK(cudaMemcpyAsync(out16, b->moments, sizeof(double) * MOM_COUNT * b->n_cells, cudaMemcpyDeviceToHost,
                            b->stream));
   VL_CHECK(cudaStreamSynchronize(b->stream));
   return VLGPU_OK;
}

int vlgpu_batch_intersections(vlgpu_batch* b, double* out12) {
   if (!b || !out12) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   VL_CHECK(cudaMemcpyAsync(out12, b->isect12, sizeof(double) * 12 * b->n_cells, cudaMemcpyDeviceToHost, b->stream));
   VL_CHECK(cudaStreamSynchronize(b->stream));
   return VLGPU_OK;
}

int vlgpu_batch_stream(vlgpu_batch* b, void** stream) {
   if (!b || !stream) return VLGPU_EINVAL;
   *stream = (void*)b->stream;
   return VLGPU_OK;
}

int vlgpu_batch_profile(vlgpu_batch* b, int enable) {
   if (!b) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   VL_CHECK(cudaStreamSynchronize(b->stream));
   if (enable && b->prof_events.empty()) {
      b->prof_events.resize(4096);
      for (auto& ev : b->prof_events) VL_CHECK(cudaEventCreate(&ev));
   }
   b->profiling = enable != 0;
   b->prof_used = 0;
   return VLGPU_OK;
}

int vlgpu_batch_stats(vlgpu_batch* b, uint64_t* out8) {
   if (!b || !out8) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   VL_CHECK(cudaStreamSynchronize(b->stream));
   BatchStats st{};
   VL_CHECK(cudaMemcpy(&st, b->stats, sizeof(st), cudaMemcpyDeviceToHost));
   double ms = 0.0;
   for (size_t q = 0; q + 1 < b->prof_used; q += 2) {
      float t = 0.f;
      VL_CHECK(cudaEventElapsedTime(&t, b->prof_events[q], b->prof_events[q + 1]));
      ms += t;
   }
   out8[0] = b->launches;
   out8[1] = st.sweeps;
   out8[2] = st.src_blocks;
   out8[3] = st.dst_blocks;
   out8[4] = b->remap_launches;
   out8[5] = (uint64_t)(ms * 1e6);
   out8[6] = b->prof_used / 2;
   out8[7] = st.sets;
   return VLGPU_OK;
}

int vlgpu_batch_stats2(vlgpu_batch* b, uint64_t* out) {
   if (!b || !out) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   VL_CHECK(cudaStreamSynchronize(b->stream));
   BatchStats st{};
   VL_CHECK(cudaMemcpy(&st, b->stats, sizeof(st), cudaMemcpyDeviceToHost));
   out[0] = st.step_blocks;
   return VLGPU_OK;
}

int vlgpu_batch_set_grid(vlgpu_batch* b, const uint32_t dims[3], const double dx[3]) {
   if (!b || !dims || !dx) return VLGPU_EINVAL;
   if ((uint64_t)dims[0] * dims[1] * dims[2] != b->n_cells) return VLGPU_EINVAL;
   for (int d = 0; d < 3; ++d)
      if (dims[d] == 0 || dims[d] > TR_MAX_N || !(dx[d] > 0.0)) return VLGPU_EINVAL;
   if (union_words(b->mdev) > 12288) return VLGPU_EINVAL;  // union bitmap and prefix fit in 96 KB
   VL_CHECK(cudaSetDevice(b->device));
   VL_CHECK(cudaStreamSynchronize(b->stream));
   if (!b->item_gid) {
      const uint64_t cap = b->capacity;
      b->row_cap = 4 * cap;
      VL_CHECK(cudaMalloc(&b->item_gid, sizeof(uint32_t) * cap));
      VL_CHECK(cudaMalloc(&b->item_pencil, sizeof(uint32_t) * cap));
      VL_CHECK(cudaMalloc(&b->trans_rows, sizeof(uint32_t) * b->row_cap));
      VL_CHECK(cudaMalloc(&b->trans_src, sizeof(uint32_t) * b->row_cap));
      // content masks of the adjustment: room for 512 rows per cell on average
      const uint64_t words = std::min<uint64_t>(3ull * 512 * b->n_cells, 0xfffffff0ull);
      b->mask_cap = (uint32_t)words;
      VL_CHECK(cudaMalloc(&b->mask_recs, sizeof(MaskRec) * b->n_cells));
      VL_CHECK(cudaMalloc(&b->mask_pool, sizeof(uint32_t) * words));
      VL_CHECK(cudaMalloc(&b->mask_top, sizeof(uint32_t)));
      VL_CHECK(cudaMalloc(&b->tcounters, sizeof(TransCounters)));
      VL_CHECK(cudaMemset(b->tcounters, 0, sizeof(TransCounters)));
   }
   // the 26 nearest neighbours of every cell, periodic, the cell itself excluded
   std::vector<int32_t> nb((size_t)b->n_cells * 26);
   for (uint32_t c = 0; c < b->n_cells; ++c) {
      const int x = (int)(c % dims[0]), y = (int)((c / dims[0]) % dims[1]), z = (int)(c / (dims[0] * dims[1]));
      int q = 0;
      for (int dz = -1; dz <= 1; ++dz)
         for (int dy = -1; dy <= 1; ++dy)
            for (int dx_ = -1; dx_ <= 1; ++dx_) {
               if (dx_ == 0 && dy == 0 && dz == 0) continue;
               const int xx = (x + dx_ + (int)dims[0]) % (int)dims[0];
               const int yy = (y + dy + (int)dims[1]) % (int)dims[1];
               const int zz = (z + dz + (int)dims[2]) % (int)dims[2];
               const uint32_t n = (uint32_t)xx + dims[0] * ((uint32_t)yy + dims[1] * (uint32_t)zz);
               nb[(size_t)c * 26 + q++] = (n == c) ? -1 : (int32_t)n;
            }
   }
   if (!b->neighbors) VL_CHECK(cudaMalloc(&b->neighbors, sizeof(int32_t) * nb.size()));
   if (!b->dt_buf) VL_CHECK(cudaMalloc(&b->dt_buf, sizeof(double) * 2 * b->n_cells));
   if (!b->moments_r) {
      VL_CHECK(cudaMalloc(&b->moments_r, sizeof(double) * MOM_COUNT * b->n_cells));
      VL_CHECK(cudaMemset(b->moments_r, 0, sizeof(double) * MOM_COUNT * b->n_cells));
   }
   VL_CHECK(cudaMemcpy(b->neighbors, nb.data(), sizeof(int32_t) * nb.size(), cudaMemcpyHostToDevice));
   for (int d = 0; d < 3; ++d) {
      b->grid_dims[d] = dims[d];
      b->grid_dx[d] = dx[d];
   }
   b->has_grid = true;
   return VLGPU_OK;
}

int vlgpu_translate(vlgpu_batch* b, uint32_t dimension, double dt) {
   if (!b || dimension > 2 || !b->has_grid) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   return translate_device(b, dimension, dt);
}

int vlgpu_vlasov_step(vlgpu_batch* b, const vlgpu_cell_fields* fields, double dt, uint32_t map_order) {
   if (!b || !fields || map_order > 2 || !b->has_grid) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   const std::vector<double> dts(b->n_cells, dt);
   const int st = stage_fields(b, fields, dts.data());
   if (st != VLGPU_OK) return st;
   return vlasov_step_device(b, dt, map_order);
}

int vlgpu_vlasov_step_device(vlgpu_batch* b, double dt, uint32_t map_order) {
   if (!b || map_order > 2 || !b->has_grid) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   return vlasov_step_device(b, dt, map_order);
}

int vlgpu_batch_moments_r(vlgpu_batch* b, double* out16) {
   if (!b || !out16 || !b->moments_r) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   VL_CHECK(cudaMemcpyAsync(out16, b->moments_r, sizeof(double) * MOM_COUNT * b->n_cells, cudaMemcpyDeviceToHost,
                            b->stream));
   VL_CHECK(cudaStreamSynchronize(b->stream));
   return VLGPU_OK;
}

int vlgpu_batch_fill_maxwellian(vlgpu_batch* b, const vlgpu_maxwellian* cells) {
   if (!b || !cells) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   const double K_B = 1.3806503e-23, PI = 3.14159265358979323846;
   const double m = b->params.mass, mv = b->params.min_value;
   std::vector<FillCell> fc(b->n_cells);
   uint64_t total = 0;
   for (uint32_t c = 0; c < b->n_cells; ++c) {
      const vlgpu_maxwellian& w = cells[c];
      FillCell& f = fc[c];
      f.n = w.n;
      bool identity = true;
      for (int q = 0; q < 9; ++q) {
         f.frame[q] = w.frame[q];
         identity &= w.frame[q] == ((q % 4 == 0) ? 1.0 : 0.0);
      }
      for (int d = 0; d < 3; ++d) {
         f.T[d] = w.T[d];
         f.V[d] = w.V[d];
         if (!(w.T[d] > 0.0)) return VLGPU_EINVAL;
      }
      f.isotropic = (identity && w.T[0] == w.T[1] && w.T[1] == w.T[2]) ? 1u : 0u;
      // candidate box: one block beyond the radius where the density can reach
      // min_value (as the projects' search does)
      const double Tmax = std::max(w.T[0], std::max(w.T[1], w.T[2]));
      const double peak = f.isotropic ? w.n * std::pow(m / (2.0 * PI * K_B * Tmax), 1.5)
                                      : w.n * std::pow(m / (2.0 * PI * K_B), 1.5) / std::sqrt(w.T[0] * w.T[1] * w.T[2]);
      const double radius = (peak <= mv) ? 0.0 : std::sqrt(2.0 * K_B * Tmax / m * std::log(peak / mv));
      bool empty = !(w.n > 0.0) || peak <= mv;
      for (int d = 0; d < 3; ++d) {
         int lo = (int)std::floor((w.V[d] - radius - b->vmin_d[d]) / b->bs_d[d]) - 1;
         int hi = (int)std::floor((w.V[d] + radius - b->vmin_d[d]) / b->bs_d[d]) + 1;
         lo = std::min(std::max(lo, 0), (int)b->mesh.len[d] - 1);
         hi = std::min(std::max(hi, 0), (int)b->mesh.len[d] - 1);
         f.lo[d] = lo;
         f.hi[d] = empty ? lo - 1 : hi;
      }
      f.row = (uint32_t)total;
      if (!empty) total += (uint64_t)(f.hi[0] - f.lo[0] + 1) * (f.hi[1] - f.lo[1] + 1) * (f.hi[2] - f.lo[2] + 1);
      if (total > b->capacity) return VLGPU_ENOMEM;
   }
   FillCell* d_cells = nullptr;
   VL_CHECK(cudaStreamSynchronize(b->stream));
   VL_CHECK(cudaMalloc(&d_cells, sizeof(FillCell) * b->n_cells));
   cudaError_t e = cudaMemcpy(d_cells, fc.data(), sizeof(FillCell) * b->n_cells, cudaMemcpyHostToDevice);
   if (e == cudaSuccess)
      e = launch_fill(d_cells, b->n_cells, b->mdev, b->vmin_d, b->bs_d, b->dv_d, m, b->gids[0], b->data[0],
                      b->slots[0], b->stream);
   if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
   cudaFree(d_cells);
   VL_CHECK(e);
   b->launches += 1;
   const uint32_t used = (uint32_t)total;
   VL_CHECK(cudaMemcpy(b->rows_used, &used, sizeof(uint32_t), cudaMemcpyHostToDevice));
   VL_CHECK(cudaMemset(b->status, 0, sizeof(uint32_t) * b->n_cells));
   set_direct_state(b, 0);
   b->content_valid = false;
   // the first block adjustment prunes the candidates (grid.cpp:289)
   const int st = adjust_device(b);
   if (st != VLGPU_OK) return st;
   VL_CHECK(cudaMemsetAsync(b->loss, 0, sizeof(double) * b->n_cells, b->stream));
   return VLGPU_OK;
}

int vlgpu_batch_interpolated_moments(vlgpu_batch* b, double* out16) {
   if (!b || !out16 || !b->moments_r) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   std::vector<double> r((size_t)MOM_COUNT * b->n_cells);
   VL_CHECK(cudaMemcpyAsync(r.data(), b->moments_r, sizeof(double) * r.size(), cudaMemcpyDeviceToHost, b->stream));
   VL_CHECK(cudaMemcpyAsync(out16, b->moments, sizeof(double) * r.size(), cudaMemcpyDeviceToHost, b->stream));
   VL_CHECK(cudaStreamSynchronize(b->stream));
   for (size_t q = 0; q < r.size(); ++q) out16[q] = 0.5 * (r[q] + out16[q]);
   return VLGPU_OK;
}

int vlgpu_batch_max_dt(vlgpu_batch* b, double max_rotation_deg, double* r_dt, double* v_dt) {
   if (!b || !r_dt || !v_dt || !b->has_grid) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   double* d = b->dt_buf;
   cudaError_t e = launch_max_dt(b->st_gids, b->st_slots, b->accel_in, b->mdev, b->vmin_d, b->bs_d, b->dv_d,
                                 b->grid_dx, b->params.charge, b->params.mass, max_rotation_deg, d, d + b->n_cells,
                                 b->n_cells, b->stream);
   if (e == cudaSuccess) e = cudaMemcpyAsync(r_dt, d, sizeof(double) * b->n_cells, cudaMemcpyDeviceToHost, b->stream);
   if (e == cudaSuccess)
      e = cudaMemcpyAsync(v_dt, d + b->n_cells, sizeof(double) * b->n_cells, cudaMemcpyDeviceToHost, b->stream);
   if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
   return cuda_status(e, "vlgpu_batch_max_dt");
}

int vlgpu_batch_capture(vlgpu_batch* b, int slot, int kind, uint32_t n_steps, const uint32_t* map_orders,
                        double dt) {
   if (!b || slot < 0 || slot >= 8 || (kind != 0 && kind != 1) || n_steps == 0 || n_steps % 2 != 0 ||
       n_steps > 6 || !map_orders || b->profiling)
      return VLGPU_EINVAL;
   if (kind == 1 && !b->has_grid) return VLGPU_EINVAL;
   for (uint32_t q = 0; q < n_steps; ++q)
      if (map_orders[q] > 2) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   VL_CHECK(cudaStreamSynchronize(b->stream));
   vlgpu_batch::GraphSlot& g = b->graphs[slot];
   if (g.exec) {
      VL_CHECK(cudaGraphExecDestroy(g.exec));
      g.exec = nullptr;
   }
   const vlgpu_batch::GraphSlot start{nullptr,      b->st_gids,     b->st_src, b->st_slots, b->cur,
                                      b->adj_next,  b->pivot_valid, false,     0,           0};
   const bool content_valid = b->content_valid;
   const unsigned long long l0 = b->launches, r0 = b->remap_launches;
   VL_CHECK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed));
   int st = VLGPU_OK;
   for (uint32_t q = 0; q < n_steps && st == VLGPU_OK; ++q)
      st = kind == 0 ? accelerate_device(b, map_orders[q], false) : vlasov_step_device(b, dt, map_orders[q]);
   cudaGraph_t graph = nullptr;
   const cudaError_t ec = cudaStreamEndCapture(b->stream, &graph);
   // nothing ran: the host's view of the buffers is the one before the capture
   const bool same_buffers = b->st_gids == start.st_gids && b->st_src == start.st_src &&
                             b->st_slots == start.st_slots && b->cur == start.cur && b->adj_next == start.adj_next;
   b->st_gids = start.st_gids;
   b->st_src = start.st_src;
   b->st_slots = start.st_slots;
   b->cur = start.cur;
   b->adj_next = start.adj_next;
   b->content_valid = content_valid;
   const bool pivot_end = b->pivot_valid;
   b->pivot_valid = start.pivot_valid;
   const unsigned long long dl = b->launches - l0, dr = b->remap_launches - r0;
   b->launches = l0;
   b->remap_launches = r0;
   if (st != VLGPU_OK) {
      if (graph) cudaGraphDestroy(graph);
      return st;
   }
   VL_CHECK(ec);
   if (!same_buffers) {
      cudaGraphDestroy(graph);
      return VLGPU_EINVAL;
   }
   cudaGraphExec_t exec = nullptr;
   const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
   cudaGraphDestroy(graph);
   VL_CHECK(ei);
   g = start;
   g.exec = exec;
   g.pivot_valid_end = pivot_end;
   g.launches = dl;
   g.remap_launches = dr;
   return VLGPU_OK;
}

int vlgpu_batch_replay(vlgpu_batch* b, int slot) {
   if (!b || slot < 0 || slot >= 8 || !b->graphs[slot].exec) return VLGPU_EINVAL;
   const vlgpu_batch::GraphSlot& g = b->graphs[slot];
   if (b->st_gids != g.st_gids || b->st_src != g.st_src || b->st_slots != g.st_slots || b->cur != g.cur ||
       b->adj_next != g.adj_next || (g.pivot_valid && !b->pivot_valid))
      return VLGPU_EINVAL;  // the batch is not in the state the graph was captured in
   VL_CHECK(cudaSetDevice(b->device));
   VL_CHECK(cudaGraphLaunch(g.exec, b->stream));
   b->launches += g.launches;
   b->remap_launches += g.remap_launches;
   b->content_valid = false;
   b->pivot_valid = g.pivot_valid_end;
   return VLGPU_OK;
}

int vlgpu_batch_set_exact(vlgpu_batch* b, int exact) {
   if (!b || (exact && b->recon != VLGPU_RECON_PPM)) return VLGPU_EINVAL;
   b->exact = exact != 0;
   return VLGPU_OK;
}

int vlgpu_batch_set_reconstruction(vlgpu_batch* b, int order) {
   if (!b || (order != VLGPU_RECON_PLM && order != VLGPU_RECON_PPM && order != VLGPU_RECON_PQM)) return VLGPU_EINVAL;
   if (b->exact && order != VLGPU_RECON_PPM) return VLGPU_EINVAL;
   b->recon = order;
   return VLGPU_OK;
}

int vlgpu_batch_sync(vlgpu_batch* b) {
   if (!b) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   VL_CHECK(cudaStreamSynchronize(b->stream));
   SweepCounters c{};
   VL_CHECK(cudaMemcpy(&c, b->counters, sizeof(c), cudaMemcpyDeviceToHost));
   if (c.overflow) return VLGPU_ENOMEM;
   if (b->tcounters) {
      TransCounters t{};
      VL_CHECK(cudaMemcpy(&t, b->tcounters, sizeof(t), cudaMemcpyDeviceToHost));
      if (t.overflow) return VLGPU_ENOMEM;
   }
   return VLGPU_OK;
}

}  // extern "C"
