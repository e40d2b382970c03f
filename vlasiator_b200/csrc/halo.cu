// Packing and unpacking the blocks of some cells of a batch, on the device,
// for the ghost-layer exchange of a spatial grid split over several batches
// (one per GPU and rank).  No reference counterpart as an entry point: it is
// the data movement of update_remote_mapping_contribution_amr and the dccrg
// remote-neighbour updates (vlasovsolver/cpu_trans_map_amr.cpp:493-810),
// rebuilt as a pack into a caller's device buffer, a transfer the caller
// makes (NCCL send/recv, or any other), and an unpack into the receiving
// batch.
#include "batch_internal.cuh"

namespace vlgpu {

// One CTA per selected cell: its blocks (IDs and 64 values) to dst_off.
__global__ void pack_cells_kernel(const uint32_t* __restrict__ gids, const float4* __restrict__ data,
                                  const uint32_t* __restrict__ desc, uint32_t* __restrict__ out_gids,
                                  float4* __restrict__ out_data) {
   const uint32_t src = desc[3 * blockIdx.x], dst = desc[3 * blockIdx.x + 1], n = desc[3 * blockIdx.x + 2];
   for (uint32_t b = threadIdx.x; b < n; b += blockDim.x) out_gids[dst + b] = gids[src + b];
   for (uint32_t q = threadIdx.x; q < 16 * n; q += blockDim.x) out_data[16 * (size_t)dst + q] = data[16 * (size_t)src + q];
}

// Every block ID below max_gid; a bad one sets *bad.
__global__ void check_gids_range_kernel(const uint32_t* __restrict__ gids, uint64_t n, uint32_t max_gid,
                                        uint32_t* __restrict__ bad) {
   for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
      if (gids[i] >= max_gid) *bad = 1u;
}

}  // namespace vlgpu

using namespace vlgpu;
using namespace vlgpu_batch_ops;

namespace {

// The batch's current state made direct (list entry p holds data row p of
// the current pool), and its cell slots and rows in use on the host.
int direct_state_slots(vlgpu_batch* b, std::vector<CellSlot>& slots, uint32_t rows[4]) {
   const int st = materialize_async(b);
   if (st != VLGPU_OK) return st;
   slots.resize(b->n_cells);
   VL_CHECK(cudaMemcpyAsync(slots.data(), b->st_slots, sizeof(CellSlot) * b->n_cells, cudaMemcpyDeviceToHost,
                            b->stream));
   VL_CHECK(cudaMemcpyAsync(rows, b->rows_used, sizeof(uint32_t) * 4, cudaMemcpyDeviceToHost, b->stream));
   VL_CHECK(cudaStreamSynchronize(b->stream));
   return VLGPU_OK;
}

// Room for n uint32 words of the per-batch exchange scratch.
int halo_scratch(vlgpu_batch* b, size_t n) {
   if (n <= b->halo_words) return VLGPU_OK;
   cudaFree(b->halo_scratch);
   b->halo_scratch = nullptr;
   b->halo_words = 0;
   VL_CHECK(cudaMalloc(&b->halo_scratch, sizeof(uint32_t) * n));
   b->halo_words = n;
   return VLGPU_OK;
}

}  // namespace

extern "C" {

int vlgpu_batch_pack_cells(vlgpu_batch* b, uint32_t n_sel, const uint32_t* cells, uint32_t* counts, uint32_t* gids,
                           float* data, uint64_t capacity, uint64_t* used) {
   if (!b || !used || (n_sel > 0 && (!cells || !counts))) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   std::vector<CellSlot> slots;
   uint32_t rows[4];
   int st = direct_state_slots(b, slots, rows);
   if (st != VLGPU_OK) return st;
   std::vector<uint32_t> desc(3 * (size_t)n_sel);
   uint64_t total = 0;
   for (uint32_t i = 0; i < n_sel; ++i) {
      if (cells[i] >= b->n_cells) return VLGPU_EINVAL;
      const CellSlot s = slots[cells[i]];
      desc[3 * i] = s.off;
      desc[3 * i + 1] = (uint32_t)total;
      desc[3 * i + 2] = s.count;
      counts[i] = s.count;
      total += s.count;
   }
   *used = total;
   if (total > capacity) return VLGPU_ENOMEM;
   if (total > 0 && (!gids || !data)) return VLGPU_EINVAL;
   if (total == 0) return VLGPU_OK;
   st = halo_scratch(b, desc.size());
   if (st != VLGPU_OK) return st;
   VL_CHECK(cudaMemcpyAsync(b->halo_scratch, desc.data(), sizeof(uint32_t) * desc.size(), cudaMemcpyHostToDevice,
                            b->stream));
   pack_cells_kernel<<<n_sel, 256, 0, b->stream>>>(b->st_gids, reinterpret_cast<const float4*>(b->data[b->cur]),
                                                   b->halo_scratch, gids, reinterpret_cast<float4*>(data));
   b->launches += 1;
   VL_CHECK(cudaGetLastError());
   VL_CHECK(cudaStreamSynchronize(b->stream));
   return VLGPU_OK;
}

int vlgpu_batch_unpack_cells(vlgpu_batch* b, uint32_t n_sel, const uint32_t* cells, const uint32_t* counts,
                             const uint32_t* gids, const float* data) {
   if (!b || (n_sel > 0 && (!cells || !counts))) return VLGPU_EINVAL;
   VL_CHECK(cudaSetDevice(b->device));
   uint64_t total = 0;
   for (uint32_t i = 0; i < n_sel; ++i) {
      if (cells[i] >= b->n_cells) return VLGPU_EINVAL;
      total += counts[i];
   }
   if (total > 0 && (!gids || !data)) return VLGPU_EINVAL;
   std::vector<CellSlot> slots;
   uint32_t rows[4];
   int st = direct_state_slots(b, slots, rows);
   if (st != VLGPU_OK) return st;
   const uint64_t L = rows[b->st_list];
   if (L + total > b->capacity) return VLGPU_ENOMEM;
   if (total > 0) {
      // the blocks' IDs must lie on the batch's mesh
      st = halo_scratch(b, 1);
      if (st != VLGPU_OK) return st;
      VL_CHECK(cudaMemsetAsync(b->halo_scratch, 0, sizeof(uint32_t), b->stream));
      const uint32_t max_gid = b->mesh.len[0] * b->mesh.len[1] * b->mesh.len[2];
      check_gids_range_kernel<<<b->sm_count * 2, 256, 0, b->stream>>>(gids, total, max_gid, b->halo_scratch);
      b->launches += 1;
      VL_CHECK(cudaGetLastError());
      uint32_t bad = 0;
      VL_CHECK(cudaMemcpyAsync(&bad, b->halo_scratch, sizeof(uint32_t), cudaMemcpyDeviceToHost, b->stream));
      VL_CHECK(cudaStreamSynchronize(b->stream));
      if (bad) return VLGPU_EINVAL;
      // appended behind the rows in use of the current list and pool; the
      // cells' earlier rows become unreferenced (the next sweep compacts)
      VL_CHECK(cudaMemcpyAsync(const_cast<uint32_t*>(b->st_gids) + L, gids, sizeof(uint32_t) * total,
                               cudaMemcpyDeviceToDevice, b->stream));
      VL_CHECK(cudaMemcpyAsync(b->data[b->cur] + L * WID3, data, sizeof(float) * WID3 * total,
                               cudaMemcpyDeviceToDevice, b->stream));
   }
   uint64_t o = L;
   for (uint32_t i = 0; i < n_sel; ++i) {
      slots[cells[i]] = CellSlot{(uint32_t)o, counts[i]};
      o += counts[i];
   }
   rows[b->st_list] = (uint32_t)(L + total);
   rows[b->cur] = (uint32_t)(L + total);
   VL_CHECK(cudaMemcpyAsync(const_cast<CellSlot*>(b->st_slots), slots.data(), sizeof(CellSlot) * b->n_cells,
                            cudaMemcpyHostToDevice, b->stream));
   VL_CHECK(cudaMemcpyAsync(b->rows_used, rows, sizeof(uint32_t) * 4, cudaMemcpyHostToDevice, b->stream));
   VL_CHECK(cudaStreamSynchronize(b->stream));
   b->content_valid = false;
   b->pivot_valid = false;
   return VLGPU_OK;
}

}  // extern "C"
