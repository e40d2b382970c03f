// Serving engine: a request loop around one device-resident batch.
//
// Independent VDF-advance requests (one spatial cell each: a sparse VDF, its
// fields, a time step and a number of acceleration steps) are queued on the
// host, admitted into free cells of the batch while the block budget derived
// from the HBM budget allows, advanced together one acceleration step per
// tick (continuous batching: requests join and leave between ticks), and
// copied back when their last step is done.  A request's cell keeps its
// blocks on the device for its whole life.
//
// Every request's result is independent of the mix it ran in: cells never
// interact, block adjustment has no spatial neighbours here, and requests are
// admitted only on ticks that are multiples of three, so that step s of every
// request uses dimension order s mod 3 (the reference draws the order from the
// time step, vlasovmover.cpp:421-426).
#include <deque>
#include <unordered_map>

#include "batch_internal.cuh"

namespace vlgpu {
cudaError_t launch_materialize(const uint32_t* src_index, const float* src, float* dst, uint64_t n_blocks,
                               cudaStream_t stream);
}

namespace {

// Device bytes per block of a batch: two data pools, two sweep lists, two
// adjustment lists (IDs and data indices), the permutation, the column sets
// and the content flags.
constexpr uint64_t BYTES_PER_BLOCK = 2 * 256 + 2 * 4 + 2 * 8 + 4 + sizeof(vlgpu::ColumnSet) + 1;
// Admission keeps the live blocks below this fraction of the capacity, which
// leaves room for the blocks a step adds and for the rows of new requests.
constexpr double ADMIT_FRACTION = 0.6;

struct Request {
   std::vector<uint32_t> gids;
   std::vector<float> data;
   vlgpu_cell_fields fields{};
   double dt = 0.0;
   uint32_t steps = 0;
   uint32_t remaining = 0;
   int cell = -1;
   bool done = false;
   uint32_t status = 0;
   double rho_loss = 0.0;
   std::vector<uint32_t> out_gids;
   std::vector<float> out_data;
};

}  // namespace

struct vlgpu_server {
   vlgpu_batch* b = nullptr;
   uint64_t next_id = 1;
   uint64_t tick = 0;
   std::deque<uint64_t> pending;
   std::unordered_map<uint64_t, Request> requests;
   std::vector<int64_t> cell_request;    // request id per cell, -1 when free
   std::vector<vlgpu_cell_fields> fields;  // host mirror of every cell's fields
   std::vector<double> dts;                // and time step (0 for a free cell)
   unsigned long long completed = 0;
   unsigned long long steps_run = 0;
};

using namespace vlgpu_batch_ops;

namespace {

// Copies the finished request in `cell` back to the host and frees the cell.
int retire(vlgpu_server* s, int cell, const CellSlot& slot, const uint32_t* status, const double* loss,
           uint64_t& stage_row) {
   vlgpu_batch* b = s->b;
   Request& r = s->requests[(uint64_t)s->cell_request[cell]];
   r.out_gids.resize(slot.count);
   r.out_data.resize((size_t)slot.count * WID3);
   if (slot.count > 0) {
      VL_CHECK(cudaMemcpyAsync(r.out_gids.data(), b->st_gids + slot.off, sizeof(uint32_t) * slot.count,
                               cudaMemcpyDeviceToHost, b->stream));
      const float* src = b->data[b->cur] + (size_t)slot.off * WID3;
      if (b->st_src) {
         // gather the cell's rows into the other pool, which is free between steps
         float* staged = b->data[1 - b->cur] + (size_t)stage_row * WID3;
         VL_CHECK(launch_materialize(b->st_src + slot.off, b->data[b->cur], staged, slot.count, b->stream));
         src = staged;
         stage_row += slot.count;
      }
      VL_CHECK(cudaMemcpyAsync(r.out_data.data(), src, sizeof(float) * WID3 * slot.count, cudaMemcpyDeviceToHost,
                               b->stream));
   }
   r.status = status[cell];
   r.rho_loss = loss[cell];
   r.done = true;
   r.cell = -1;
   s->cell_request[cell] = -1;
   s->completed += 1;
   return VLGPU_OK;
}

}  // namespace

extern "C" {

int vlgpu_server_create(const vlgpu_mesh* mesh, const vlgpu_params* params, uint32_t max_cells,
                        uint64_t hbm_budget_bytes, int device, vlgpu_server** out) {
   if (!out || max_cells == 0 || hbm_budget_bytes < BYTES_PER_BLOCK * 4096) return VLGPU_EINVAL;
   uint64_t capacity = hbm_budget_bytes / BYTES_PER_BLOCK;
   if (capacity >= 0xffffffffull) capacity = 0xfffffffeull;
   vlgpu_batch* b = nullptr;
   const int st = vlgpu_batch_create(mesh, params, max_cells, capacity, device, &b);
   if (st != VLGPU_OK) return st;
   vlgpu_server* s = new vlgpu_server();
   s->b = b;
   s->cell_request.assign(max_cells, -1);
   s->fields.assign(max_cells, vlgpu_cell_fields{});
   s->dts.assign(max_cells, 0.0);
   // every cell starts empty
   std::vector<uint64_t> offs(max_cells + 1, 0);
   const int up = vlgpu_batch_upload(b, offs.data(), nullptr, nullptr);
   if (up != VLGPU_OK) {
      vlgpu_batch_destroy(b);
      delete s;
      return up;
   }
   *out = s;
   return VLGPU_OK;
}

int vlgpu_server_destroy(vlgpu_server* s) {
   if (!s) return VLGPU_EINVAL;
   vlgpu_batch_destroy(s->b);
   delete s;
   return VLGPU_OK;
}

int vlgpu_server_submit(vlgpu_server* s, uint32_t n_blocks, const uint32_t* gids, const float* data,
                        const vlgpu_cell_fields* fields, double dt, uint32_t n_steps, uint64_t* request_id) {
   if (!s || !fields || !request_id || n_steps == 0 || (n_blocks > 0 && (!gids || !data))) return VLGPU_EINVAL;
   const uint32_t maxgid = s->b->mesh.len[0] * s->b->mesh.len[1] * s->b->mesh.len[2];
   for (uint32_t q = 0; q < n_blocks; ++q)
      if (gids[q] >= maxgid) return VLGPU_EINVAL;
   if (n_blocks > ADMIT_FRACTION * (double)s->b->capacity) return VLGPU_ENOMEM;  // could never be admitted
   const uint64_t id = s->next_id++;
   Request& r = s->requests[id];
   r.gids.assign(gids, gids + n_blocks);
   r.data.assign(data, data + (size_t)n_blocks * WID3);
   r.fields = *fields;
   r.dt = dt;
   r.steps = n_steps;
   r.remaining = n_steps;
   s->pending.push_back(id);
   *request_id = id;
   return VLGPU_OK;
}

int vlgpu_server_tick(vlgpu_server* s, uint32_t* n_active, uint32_t* n_pending, uint32_t* n_done) {
   if (!s) return VLGPU_EINVAL;
   vlgpu_batch* b = s->b;
   VL_CHECK(cudaSetDevice(b->device));
   VL_CHECK(cudaStreamSynchronize(b->stream));  // the previous step is complete
   const uint32_t nc = b->n_cells;
   std::vector<CellSlot> slots(nc);
   std::vector<uint32_t> status(nc);
   std::vector<double> loss(nc);
   uint32_t rows[4];
   VL_CHECK(cudaMemcpyAsync(slots.data(), b->st_slots, sizeof(CellSlot) * nc, cudaMemcpyDeviceToHost, b->stream));
   VL_CHECK(cudaMemcpyAsync(status.data(), b->status, sizeof(uint32_t) * nc, cudaMemcpyDeviceToHost, b->stream));
   VL_CHECK(cudaMemcpyAsync(loss.data(), b->loss, sizeof(double) * nc, cudaMemcpyDeviceToHost, b->stream));
   VL_CHECK(cudaMemcpyAsync(rows, b->rows_used, sizeof(rows), cudaMemcpyDeviceToHost, b->stream));
   VL_CHECK(cudaStreamSynchronize(b->stream));

   // 1. retire the requests whose last step is done
   uint32_t done_now = 0;
   uint64_t stage_row = 0;
   bool slots_changed = false;
   for (uint32_t c = 0; c < nc; ++c) {
      const int64_t id = s->cell_request[c];
      if (id < 0 || s->requests[(uint64_t)id].remaining > 0) continue;
      const int st = retire(s, (int)c, slots[c], status.data(), loss.data(), stage_row);
      if (st != VLGPU_OK) return st;
      slots[c] = CellSlot{0u, 0u};
      s->dts[c] = 0.0;
      ++done_now;
      slots_changed = true;
   }

   // 2. admit pending requests (on ticks that are multiples of three)
   uint64_t live = 0;
   for (uint32_t c = 0; c < nc; ++c)
      if (s->cell_request[c] >= 0) live += slots[c].count;
   uint64_t L = rows[b->st_list];
   uint64_t D = b->st_src ? rows[b->cur] : L;
   std::vector<uint32_t> admitted;
   if (s->tick % 3 == 0) {
      uint32_t c = 0;
      while (!s->pending.empty()) {
         Request& r = s->requests[s->pending.front()];
         const uint64_t n = r.gids.size();
         if ((double)(live + n) > ADMIT_FRACTION * (double)b->capacity || L + n > b->capacity ||
             D + n > b->capacity)
            break;
         while (c < nc && s->cell_request[c] >= 0) ++c;
         if (c == nc) break;
         const uint64_t id = s->pending.front();
         s->pending.pop_front();
         s->cell_request[c] = (int64_t)id;
         r.cell = (int)c;
         if (n > 0) {
            VL_CHECK(cudaMemcpyAsync(const_cast<uint32_t*>(b->st_gids) + L, r.gids.data(), sizeof(uint32_t) * n,
                                     cudaMemcpyHostToDevice, b->stream));
            VL_CHECK(cudaMemcpyAsync(b->data[b->cur] + D * WID3, r.data.data(), sizeof(float) * WID3 * n,
                                     cudaMemcpyHostToDevice, b->stream));
         }
         if (b->st_src && n > 0) {
            std::vector<uint32_t> idx(n);
            for (uint64_t q = 0; q < n; ++q) idx[q] = (uint32_t)(D + q);
            VL_CHECK(cudaMemcpyAsync(const_cast<uint32_t*>(b->st_src) + L, idx.data(), sizeof(uint32_t) * n,
                                     cudaMemcpyHostToDevice, b->stream));
         }
         // copies from pageable memory return once the source has been staged
         std::vector<uint32_t>().swap(r.gids);
         std::vector<float>().swap(r.data);
         slots[c] = CellSlot{(uint32_t)L, (uint32_t)n};
         s->fields[c] = r.fields;
         s->dts[c] = r.dt;
         status[c] = 0;
         loss[c] = 0.0;
         admitted.push_back(c);
         L += n;
         D += n;
         live += n;
         slots_changed = true;
      }
   }
   if (slots_changed) {
      VL_CHECK(cudaMemcpyAsync(const_cast<CellSlot*>(b->st_slots), slots.data(), sizeof(CellSlot) * nc,
                               cudaMemcpyHostToDevice, b->stream));
      rows[b->st_list] = (uint32_t)L;
      if (b->st_src) rows[b->cur] = (uint32_t)D;
      VL_CHECK(cudaMemcpyAsync(b->rows_used, rows, sizeof(rows), cudaMemcpyHostToDevice, b->stream));
      b->content_valid = false;
      if (b->pivot_valid && !admitted.empty()) {
         // the admitted cells' pivots from their VDFs; every other cell keeps
         // the pivot its last step wrote, so a request's steps do not depend
         // on the requests admitted beside it
         const int st = moments_device(b, false, b->mom_scratch);
         if (st != VLGPU_OK) return st;
         for (uint32_t c : admitted)
            VL_CHECK(cudaMemcpyAsync(b->pivot + (size_t)c * MOM_COUNT, b->mom_scratch + (size_t)c * MOM_COUNT,
                                     sizeof(double) * MOM_COUNT, cudaMemcpyDeviceToDevice, b->stream));
      }
   }
   for (uint32_t c : admitted) {
      // a new request starts with a clean status word and loss counter
      VL_CHECK(cudaMemcpyAsync(b->status + c, &status[c], sizeof(uint32_t), cudaMemcpyHostToDevice, b->stream));
      VL_CHECK(cudaMemcpyAsync(b->loss + c, &loss[c], sizeof(double), cudaMemcpyHostToDevice, b->stream));
   }

   // 3. one acceleration step of every active cell
   uint32_t active = 0;
   for (uint32_t c = 0; c < nc; ++c) active += s->cell_request[c] >= 0;
   if (active > 0) {
      int st = stage_fields(b, s->fields.data(), s->dts.data());
      if (st != VLGPU_OK) return st;
      st = accelerate_device(b, (uint32_t)(s->tick % 3), false);
      if (st != VLGPU_OK) return st;
      for (uint32_t c = 0; c < nc; ++c)
         if (s->cell_request[c] >= 0) s->requests[(uint64_t)s->cell_request[c]].remaining -= 1;
      s->steps_run += active;
   } else {
      VL_CHECK(cudaStreamSynchronize(b->stream));
   }
   s->tick += 1;
   if (n_active) *n_active = active;
   if (n_pending) *n_pending = (uint32_t)s->pending.size();
   if (n_done) *n_done = done_now;
   return VLGPU_OK;
}

int vlgpu_server_result(vlgpu_server* s, uint64_t request_id, uint32_t* n_blocks, uint32_t* gids, float* data,
                        uint64_t capacity, uint32_t* status, double* rho_loss) {
   if (!s || !n_blocks) return VLGPU_EINVAL;
   auto it = s->requests.find(request_id);
   if (it == s->requests.end()) return VLGPU_EINVAL;
   Request& r = it->second;
   if (!r.done) return VLGPU_EAGAIN;
   const uint32_t n = (uint32_t)r.out_gids.size();
   *n_blocks = n;
   if (n > capacity) return VLGPU_ENOMEM;
   if (n > 0 && (!gids || !data)) return VLGPU_EINVAL;
   // ascending global IDs, as vlgpu_batch_download returns blocks
   std::vector<uint32_t> order(n);
   for (uint32_t q = 0; q < n; ++q) order[q] = q;
   std::sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return r.out_gids[x] < r.out_gids[y]; });
   for (uint32_t q = 0; q < n; ++q) {
      gids[q] = r.out_gids[order[q]];
      std::memcpy(data + (size_t)q * WID3, r.out_data.data() + (size_t)order[q] * WID3, sizeof(float) * WID3);
   }
   if (status) *status = r.status;
   if (rho_loss) *rho_loss = r.rho_loss;
   s->requests.erase(it);
   return VLGPU_OK;
}

int vlgpu_server_stats(vlgpu_server* s, uint64_t* out4) {
   if (!s || !out4) return VLGPU_EINVAL;
   uint64_t st2 = 0;
   const int rc = vlgpu_batch_stats2(s->b, &st2);
   if (rc != VLGPU_OK) return rc;
   out4[0] = s->tick;
   out4[1] = s->completed;
   out4[2] = s->steps_run;
   out4[3] = st2 * WID3;
   return VLGPU_OK;
}

int vlgpu_server_batch(vlgpu_server* s, vlgpu_batch** batch) {
   if (!s || !batch) return VLGPU_EINVAL;
   *batch = s->b;
   return VLGPU_OK;
}

}  // extern "C"
