// Sparse velocity-block adjustment for sm_100a.
//
// Semantics of SpatialCell::adjust_velocity_blocks
// (spatial_cells/spatial_cell_cpu.cpp:179-273): the new block set is H = the
// blocks with content (any cell >= minValue, compute_block_has_content,
// spatial_cell_cpu.cpp:290-320) dilated by +-blockAddWidthV in all three
// velocity directions, clipped to the mesh, plus every block that has content
// in one of the cell's spatial neighbours (the 26 nearest cells of a periodic
// grid, Neighborhoods::NEAREST of grid.cpp:979-997), when the batch is a grid.
// Blocks with content always stay, blocks in H keep their data, blocks not
// in H are removed and their mass sum(f)*dv^3 is added to RHOLOSSADJUST,
// blocks of H that did not exist are added with zero data.
//
// Persistent CTAs of 256 threads, one cell at a time, the largest cells
// first.  The content set and H live in shared memory as 96-bit x-masks over
// the (y,z) rows of the cell's dilated bounding box.  The output
// is a new block list sorted by global ID plus, per block, the index of its
// data in the current pool (or none for an added block): no VDF value is
// copied, the next sweep reads the kept blocks where they are.
//
// On a grid, content_mask_kernel first writes every cell's content mask once
// (its content bounding box and the x-mask rows over it, in a pool), so that
// a cell ORs its 26 neighbours' mask rows instead of walking their block
// lists; a cell whose mask did not fit (box too large, pool full) is read from
// its list as before.
#include <cstdint>

#include "moments_record.cuh"
#include "vlgpu_common.cuh"

namespace vlgpu {

constexpr int ADJ_THREADS = 256;
constexpr int ADJ_MIN_CTAS = 3;   // CTAs per SM the register budget is set for
constexpr int ADJ_UNROLL = 4;     // list entries per thread in flight
constexpr uint32_t ADJ_QUEUE = 32 * ADJ_UNROLL;  // old blocks a warp queues per pass
constexpr uint32_t ADJ_KEPT = 0x80000000u;       // queue flag: the block stays
constexpr uint32_t NO_BLOCK = 0xffffffffu;

__device__ __forceinline__ uint32_t adj_exclusive_scan(uint32_t v, uint32_t* warp_sums, uint32_t& total) {
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   uint32_t x = v;
#pragma unroll
   for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
   }
   if (lane == 31) warp_sums[warp] = x;
   __syncthreads();
   if (warp == 0) {
      const int nw = blockDim.x >> 5;
      uint32_t s = (lane < nw) ? warp_sums[lane] : 0u;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
         const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
         if (lane >= o) s += y;
      }
      if (lane < nw) warp_sums[lane] = s;
   }
   __syncthreads();
   total = warp_sums[(blockDim.x >> 5) - 1];
   const uint32_t before = (warp > 0) ? warp_sums[warp - 1] : 0u;
   __syncthreads();
   return before + x - v;
}

// Content of one block: any of its 64 values >= min_value (compared in
// double, as the reference compares Realf data with the Real threshold).
__device__ __forceinline__ bool block_has_content(const float* __restrict__ blk, double min_value) {
   const float4* q = reinterpret_cast<const float4*>(blk);
   bool c = false;
   for (int i = 0; i < 16; ++i) {
      const float4 v = __ldg(q + i);
      c |= ((double)v.x >= min_value) | ((double)v.y >= min_value) | ((double)v.z >= min_value) |
           ((double)v.w >= min_value);
   }
   return c;
}

__device__ __forceinline__ uint32_t shl96(uint32_t w0, uint32_t w1, uint32_t w2, int word, int s) {
   // word `word` of the 96-bit value (w0,w1,w2) shifted left by s (0 <= s < 32)
   if (s == 0) return word == 0 ? w0 : (word == 1 ? w1 : w2);
   if (word == 0) return w0 << s;
   if (word == 1) return (w1 << s) | (w0 >> (32 - s));
   return (w2 << s) | (w1 >> (32 - s));
}
__device__ __forceinline__ uint32_t shr96(uint32_t w0, uint32_t w1, uint32_t w2, int word, int s) {
   if (s == 0) return word == 0 ? w0 : (word == 1 ? w1 : w2);
   if (word == 0) return (w0 >> s) | (w1 << (32 - s));
   if (word == 1) return (w1 >> s) | (w2 << (32 - s));
   return w2 >> s;
}

__device__ __forceinline__ bool list_block_content(const uint32_t* __restrict__ src_index,
                                                   const uint8_t* __restrict__ content,
                                                   const float* __restrict__ data, uint32_t pos, double min_value) {
   const uint32_t idx = src_index ? src_index[pos] : pos;
   if (idx == NO_BLOCK) return false;
   if (content) return content[pos] != 0;
   return block_has_content(data + (size_t)idx * WID3, min_value);
}

constexpr uint32_t NO_MASK = 0xffffffffu;
constexpr int MASK_THREADS = 256;
constexpr uint32_t MASK_SMEM_ROWS = 1600;

// One CTA per cell: the content bounding box (y, z) and, when its rows fit,
// the content x-mask rows, copied to the pool at an offset taken from
// pool_top.
__global__ void __launch_bounds__(MASK_THREADS) content_mask_kernel(
   const uint32_t* __restrict__ gids, const uint32_t* __restrict__ src_index, const CellSlot* __restrict__ slots,
   const uint8_t* __restrict__ content, const float* __restrict__ data, MeshDev mesh, double min_value,
   MaskRec* __restrict__ recs, uint32_t* __restrict__ pool, uint32_t* __restrict__ pool_top, uint32_t pool_cap) {
   __shared__ uint32_t C[3 * MASK_SMEM_ROWS];
   __shared__ int s_box[4];
   __shared__ uint32_t s_off;
   const uint32_t cell = blockIdx.x;
   const CellSlot s = slots[cell];
   if (threadIdx.x == 0) {
      s_box[0] = 1 << 20;
      s_box[1] = -1;
      s_box[2] = 1 << 20;
      s_box[3] = -1;
   }
   __syncthreads();
   {
      int y0 = 1 << 20, y1 = -1, z0 = 1 << 20, z1 = -1;
      for (uint32_t b = threadIdx.x; b < s.count; b += blockDim.x) {
         if (list_block_content(src_index, content, data, s.off + b, min_value)) {
            const uint32_t g = gids[s.off + b];
            uint32_t bx, by, bz;
            block_xyz(mesh, g, bx, by, bz);
            const int y = (int)by, z = (int)bz;
            y0 = min(y0, y); y1 = max(y1, y); z0 = min(z0, z); z1 = max(z1, z);
         }
      }
      atomicMin(&s_box[0], y0); atomicMax(&s_box[1], y1);
      atomicMin(&s_box[2], z0); atomicMax(&s_box[3], z1);
   }
   __syncthreads();
   const int y0 = s_box[0], y1 = s_box[1], z0 = s_box[2], z1 = s_box[3];
   const int ny = (y1 >= 0) ? y1 - y0 + 1 : 0, nz = (y1 >= 0) ? z1 - z0 + 1 : 0;
   const uint32_t rows = (uint32_t)(ny * nz);
   if (rows > MASK_SMEM_ROWS) {
      if (threadIdx.x == 0) recs[cell] = MaskRec{y0, y1, z0, z1, NO_MASK, {0u, 0u, 0u}};
      return;
   }
   for (uint32_t q = threadIdx.x; q < 3 * rows; q += blockDim.x) C[q] = 0u;
   __syncthreads();
   for (uint32_t b = threadIdx.x; b < s.count; b += blockDim.x) {
      if (list_block_content(src_index, content, data, s.off + b, min_value)) {
         const uint32_t g = gids[s.off + b];
         uint32_t x, by, bz;
         block_xyz(mesh, g, x, by, bz);
         const int y = (int)by, z = (int)bz;
         atomicOr(&C[3 * (uint32_t)((z - z0) * ny + (y - y0)) + (x >> 5)], 1u << (x & 31));
      }
   }
   if (threadIdx.x == 0) {
      uint32_t off = 0u;
      if (rows) {
         off = atomicAdd(pool_top, 3u * rows);
         if ((uint64_t)off + 3u * rows > pool_cap) off = NO_MASK;
      }
      s_off = off;
      recs[cell] = MaskRec{y0, y1, z0, z1, off, {0u, 0u, 0u}};
   }
   __syncthreads();
   const uint32_t off = s_off;
   if (off != NO_MASK)
      for (uint32_t q = threadIdx.x; q < 3 * rows; q += blockDim.x) pool[off + q] = C[q];
}

// One cell at a time per CTA of ADJ_THREADS threads; persistent CTAs take
// the cells from a counter in the order `order` gives (largest first), so
// the longest cells start first and the rest balance over the CTAs.  Per
// cell: the content bounding box, the content mask C (one shared-memory OR
// per content block, after the lanes of a warp that set bits of the same
// word combine them), the dilated set H row by row, the neighbours' content,
// an exclusive scan of the row counts, the GID-sorted output list, and a pass
// over the old blocks that points kept entries at their data and sums the
// removed ones (a half-warp per removed block, float4 rows).
__global__ void __launch_bounds__(ADJ_THREADS, ADJ_MIN_CTAS) adjust_kernel(
   const uint32_t* __restrict__ gids, const uint32_t* __restrict__ src_index, const CellSlot* __restrict__ slots,
   const uint8_t* __restrict__ content, const float* __restrict__ data, const int32_t* __restrict__ neighbors,
   uint32_t* __restrict__ out_gids, uint32_t* __restrict__ out_src, CellSlot* __restrict__ out_slots,
   double* __restrict__ loss, uint32_t* __restrict__ status, SweepCounters* __restrict__ counters,
   uint32_t out_capacity, MeshDev mesh, double min_value, int add_width, double dv3, uint32_t n_cells,
   uint32_t smem_rows, uint32_t* __restrict__ scratch, const MaskRec* __restrict__ masks,
   const uint32_t* __restrict__ pool, const uint32_t* __restrict__ order, double* __restrict__ mom_record,
   double* __restrict__ pivot, int write_pivot, MomentFrame fr) {
   extern __shared__ uint32_t smem[];
   __shared__ uint32_t warp_sums[32];
   __shared__ int s_box[8];
   __shared__ uint32_t s_base, s_flags, s_item;
   __shared__ double s_loss[ADJ_THREADS / 32];
   __shared__ double s_mom[ADJ_THREADS / 32][10];            // the warps' moment sums
   __shared__ uint32_t s_qidx[ADJ_THREADS / 32][ADJ_QUEUE];  // a warp's queue of old blocks: data row
   __shared__ uint32_t s_qgid[ADJ_THREADS / 32][ADJ_QUEUE];  // and block ID (| ADJ_KEPT when kept)
   __shared__ MaskRec s_rec[27];     // the neighbours' content masks (26: the cell's own)
   __shared__ uint32_t s_first[27];  // first mask-row item of each neighbour
   constexpr uint32_t FULL = 0xffffffffu;
   const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   const uint32_t L0 = mesh.len[0], L1 = mesh.len[1], L2 = mesh.len[2];
   const uint32_t xmask2 = (L0 >= 96) ? 0xffffffffu : ((L0 <= 64) ? 0u : ((1u << (L0 - 64)) - 1u));
   const uint32_t xmask1 = (L0 >= 64) ? 0xffffffffu : ((L0 <= 32) ? 0u : ((1u << (L0 - 32)) - 1u));
   const uint32_t xmask0 = (L0 >= 32) ? 0xffffffffu : ((1u << L0) - 1u);

   for (;;) {
   if (threadIdx.x == 0) {
      s_item = atomicAdd(&counters->cell_next, 1u);
      for (int q = 0; q < 8; q += 2) {
         s_box[q] = 1 << 20;
         s_box[q + 1] = -1;
      }
      s_flags = 0;
   }
   __syncthreads();
   const uint32_t item = s_item;
   if (item >= n_cells) break;
   const uint32_t cell = order[item];
   const CellSlot s = slots[cell];
   if (threadIdx.x < 27) {
      // mask records of the neighbours (a missing neighbour reads as empty)
      // and of the cell itself; without masks every list is walked
      MaskRec r{0, -1, 0, -1, NO_MASK, {0u, 0u, 0u}};
      if (masks) {
         const int32_t nc = (threadIdx.x < 26) ? (neighbors ? neighbors[(size_t)cell * 26 + threadIdx.x] : -1)
                                               : (int32_t)cell;
         r = (nc >= 0) ? masks[nc] : MaskRec{0, -1, 0, -1, 0u, {0u, 0u, 0u}};
      }
      s_rec[threadIdx.x] = r;
   }
   __syncthreads();
   // pass 1: bounding boxes (y, z) of the cell's content blocks and of its
   // spatial neighbours' content blocks (warp reductions, one shared
   // min/max per warp)
   {
      const bool own_mask = s_rec[26].off != NO_MASK;
      if (own_mask) {
         if (threadIdx.x == 0) {
            s_box[0] = s_rec[26].y0; s_box[1] = s_rec[26].y1;
            s_box[2] = s_rec[26].z0; s_box[3] = s_rec[26].z1;
         }
      } else {
         int y0 = 1 << 20, y1 = -1, z0 = 1 << 20, z1 = -1;
         for (uint32_t b0 = threadIdx.x; b0 < s.count; b0 += ADJ_THREADS * ADJ_UNROLL) {
            bool c[ADJ_UNROLL];
            uint32_t g[ADJ_UNROLL];
#pragma unroll
            for (int u = 0; u < ADJ_UNROLL; ++u) {
               const uint32_t b = b0 + ADJ_THREADS * u;
               c[u] = b < s.count && list_block_content(src_index, content, data, s.off + b, min_value);
               g[u] = b < s.count ? gids[s.off + b] : 0u;
            }
#pragma unroll
            for (int u = 0; u < ADJ_UNROLL; ++u) {
               if (!c[u]) continue;
               uint32_t bx, by, bz;
               block_xyz(mesh, g[u], bx, by, bz);
               y0 = min(y0, (int)by); y1 = max(y1, (int)by);
               z0 = min(z0, (int)bz); z1 = max(z1, (int)bz);
            }
         }
         y0 = __reduce_min_sync(FULL, y0); y1 = __reduce_max_sync(FULL, y1);
         z0 = __reduce_min_sync(FULL, z0); z1 = __reduce_max_sync(FULL, z1);
         if (lane == 0) {
            atomicMin(&s_box[0], y0); atomicMax(&s_box[1], y1);
            atomicMin(&s_box[2], z0); atomicMax(&s_box[3], z1);
         }
      }
      if (neighbors) {
         int ny0 = 1 << 20, ny1 = -1, nz0 = 1 << 20, nz1 = -1;
         if (threadIdx.x < 26 && s_rec[threadIdx.x].off != NO_MASK && s_rec[threadIdx.x].y1 >= 0) {
            const MaskRec& r = s_rec[threadIdx.x];
            ny0 = r.y0; ny1 = r.y1; nz0 = r.z0; nz1 = r.z1;
         }
         for (int q = 0; q < 26; ++q) {
            const int32_t nc = neighbors[(size_t)cell * 26 + q];
            if (nc < 0 || s_rec[q].off != NO_MASK) continue;
            const CellSlot ns = slots[nc];
            for (uint32_t b = threadIdx.x; b < ns.count; b += ADJ_THREADS) {
               if (list_block_content(src_index, content, data, ns.off + b, min_value)) {
                  uint32_t bx, by, bz;
                  block_xyz(mesh, gids[ns.off + b], bx, by, bz);
                  ny0 = min(ny0, (int)by); ny1 = max(ny1, (int)by);
                  nz0 = min(nz0, (int)bz); nz1 = max(nz1, (int)bz);
               }
            }
         }
         ny0 = __reduce_min_sync(FULL, ny0); ny1 = __reduce_max_sync(FULL, ny1);
         nz0 = __reduce_min_sync(FULL, nz0); nz1 = __reduce_max_sync(FULL, nz1);
         if (lane == 0) {
            atomicMin(&s_box[4], ny0); atomicMax(&s_box[5], ny1);
            atomicMin(&s_box[6], nz0); atomicMax(&s_box[7], nz1);
         }
      }
   }
   __syncthreads();
   const bool own_any = s_box[1] >= 0, nb_any = s_box[5] >= 0;
   const bool any = own_any || nb_any;
   int y0 = 1 << 20, y1 = -1, z0 = 1 << 20, z1 = -1;
   if (own_any) {
      y0 = max(0, s_box[0] - add_width); y1 = min((int)L1 - 1, s_box[1] + add_width);
      z0 = max(0, s_box[2] - add_width); z1 = min((int)L2 - 1, s_box[3] + add_width);
   }
   if (nb_any) {
      y0 = min(y0, s_box[4]); y1 = max(y1, s_box[5]);
      z0 = min(z0, s_box[6]); z1 = max(z1, s_box[7]);
   }
   if (!any) { y0 = 0; y1 = -1; z0 = 0; z1 = -1; }
   const int ny = y1 - y0 + 1, nz = z1 - z0 + 1;
   const uint32_t rows = any ? (uint32_t)(ny * nz) : 0u;
   // the masks live in shared memory when they fit, else in this CTA's slice
   // of a global scratch array (a full velocity plane of rows)
   uint32_t* const base = (rows <= smem_rows) ? smem : scratch + (size_t)blockIdx.x * 7 * L1 * L2;
   uint32_t* C = base;              // 3 * rows
   uint32_t* H = base + 3 * rows;   // 3 * rows
   uint32_t* prefix = base + 6 * rows;  // rows
   for (uint32_t q = threadIdx.x; q < 3 * rows; q += ADJ_THREADS) C[q] = 0;
   __syncthreads();
   // pass 2: content mask rows (copied from the cell's own mask when it has one)
   if (s_rec[26].off != NO_MASK) {
      const MaskRec& m = s_rec[26];
      if (m.y1 >= 0) {
         const int my = m.y1 - m.y0 + 1;
         const uint32_t mrows = (uint32_t)(my * (m.z1 - m.z0 + 1));
         for (uint32_t q = threadIdx.x; q < 3 * mrows; q += ADJ_THREADS) {
            const uint32_t mr = q / 3, w = q - 3 * mr;
            const int y = m.y0 + (int)(mr % my), z = m.z0 + (int)(mr / my);
            C[3 * (uint32_t)((z - z0) * ny + (y - y0)) + w] = pool[m.off + q];
         }
      }
   } else if (own_any) {
      for (uint32_t b0 = warp * 32; b0 < s.count; b0 += ADJ_THREADS * ADJ_UNROLL) {
         bool cc[ADJ_UNROLL];
         uint32_t gg[ADJ_UNROLL];
#pragma unroll
         for (int u = 0; u < ADJ_UNROLL; ++u) {
            const uint32_t b = b0 + ADJ_THREADS * u + lane;
            cc[u] = b < s.count && list_block_content(src_index, content, data, s.off + b, min_value);
            gg[u] = b < s.count ? gids[s.off + b] : 0u;
         }
#pragma unroll
         for (int u = 0; u < ADJ_UNROLL; ++u) {
            uint32_t key = 0xffffffffu, bit = 0u;
            if (cc[u]) {
               uint32_t x, by, bz;
               block_xyz(mesh, gg[u], x, by, bz);
               key = 3 * (uint32_t)(((int)bz - z0) * ny + ((int)by - y0)) + (x >> 5);
               bit = 1u << (x & 31);
            }
            // lanes that set bits of one word (a run of the list along x):
            // four or more combine them first
            const uint32_t match = __match_any_sync(FULL, key);
            const bool big = cc[u] && __popc(match) >= 4;
            if (cc[u] && !big) atomicOr(&C[key], bit);
            for (uint32_t leaders = __ballot_sync(FULL, big && (int)lane == __ffs(match) - 1); leaders;
                 leaders &= leaders - 1) {
               const int leader = __ffs(leaders) - 1;
               const bool mine = (__shfl_sync(FULL, match, leader) >> lane) & 1u;
               const uint32_t bits = __reduce_or_sync(FULL, mine ? bit : 0u);
               if ((int)lane == leader) atomicOr(&C[key], bits);
            }
         }
      }
   }
   __syncthreads();
   // dilation: H(y,z) = OR over |dy|,|dz| <= w of the row dilated along x
   const uint32_t chunk = (rows + ADJ_THREADS - 1) / ADJ_THREADS;
   const uint32_t r0 = min(rows, threadIdx.x * chunk), r1 = min(rows, r0 + chunk);
   for (uint32_t r = r0; r < r1; ++r) {
      const int yy = y0 + (int)(r % ny), zz = z0 + (int)(r / ny);
      uint32_t h0 = 0, h1 = 0, h2 = 0;
      for (int dz = -add_width; dz <= add_width; ++dz) {
         const int z = zz + dz;
         if (z < z0 || z > z1) continue;
         for (int dy = -add_width; dy <= add_width; ++dy) {
            const int y = yy + dy;
            if (y < y0 || y > y1) continue;
            const uint32_t rr = (uint32_t)((z - z0) * ny + (y - y0));
            const uint32_t c0 = C[3 * rr], c1 = C[3 * rr + 1], c2 = C[3 * rr + 2];
            h0 |= c0; h1 |= c1; h2 |= c2;
            for (int sft = 1; sft <= add_width; ++sft) {
               h0 |= shl96(c0, c1, c2, 0, sft) | shr96(c0, c1, c2, 0, sft);
               h1 |= shl96(c0, c1, c2, 1, sft) | shr96(c0, c1, c2, 1, sft);
               h2 |= shl96(c0, c1, c2, 2, sft) | shr96(c0, c1, c2, 2, sft);
            }
         }
      }
      h0 &= xmask0; h1 &= xmask1; h2 &= xmask2;
      H[3 * r] = h0; H[3 * r + 1] = h1; H[3 * r + 2] = h2;
   }
   __syncthreads();
   // blocks with content in a spatial neighbour (adjust_velocity_blocks,
   // spatial_cell_cpu.cpp:211-221)
   if (neighbors && nb_any) {
      // neighbours with a mask: one item per mask row of each neighbour (all
      // inside the box), consecutive threads on consecutive rows of the pool
      if (masks) {
         if (threadIdx.x == 0) {
            uint32_t t = 0;
            for (int q = 0; q < 26; ++q) {
               s_first[q] = t;
               const MaskRec& m = s_rec[q];
               if (m.off != NO_MASK && m.y1 >= 0) t += (uint32_t)((m.y1 - m.y0 + 1) * (m.z1 - m.z0 + 1));
            }
            s_first[26] = t;
         }
         __syncthreads();
         const uint32_t items = s_first[26];
         int q = 0;
         for (uint32_t it = threadIdx.x; it < items; it += ADJ_THREADS) {
            while (it >= s_first[q + 1]) ++q;
            const MaskRec& m = s_rec[q];
            const uint32_t mr = it - s_first[q];
            const uint32_t my = (uint32_t)(m.y1 - m.y0 + 1);
            const uint32_t mz = mr / my;
            const int y = m.y0 + (int)(mr - mz * my), z = m.z0 + (int)mz;
            const uint32_t* src = pool + m.off + 3 * mr;
            const uint32_t w0 = __ldg(src), w1 = __ldg(src + 1), w2 = __ldg(src + 2);
            uint32_t* dst = &H[3 * (uint32_t)((z - z0) * ny + (y - y0))];
            if (w0) atomicOr(dst, w0);
            if (w1) atomicOr(dst + 1, w1);
            if (w2) atomicOr(dst + 2, w2);
         }
      }
      for (int q = 0; q < 26; ++q) {
         const int32_t nc = neighbors[(size_t)cell * 26 + q];
         if (nc < 0 || s_rec[q].off != NO_MASK) continue;
         const CellSlot ns = slots[nc];
         for (uint32_t b = threadIdx.x; b < ns.count; b += ADJ_THREADS) {
            if (list_block_content(src_index, content, data, ns.off + b, min_value)) {
               uint32_t x, by, bz;
               block_xyz(mesh, gids[ns.off + b], x, by, bz);
               const uint32_t r = (uint32_t)(((int)bz - z0) * ny + ((int)by - y0));
               atomicOr(&H[3 * r + (x >> 5)], 1u << (x & 31));
            }
         }
      }
      __syncthreads();
   }
   uint32_t my_count = 0;
   for (uint32_t r = r0; r < r1; ++r) my_count += __popc(H[3 * r]) + __popc(H[3 * r + 1]) + __popc(H[3 * r + 2]);
   uint32_t total;
   uint32_t base_r = adj_exclusive_scan(my_count, warp_sums, total);
   for (uint32_t r = r0; r < r1; ++r) {
      prefix[r] = base_r;
      base_r += __popc(H[3 * r]) + __popc(H[3 * r + 1]) + __popc(H[3 * r + 2]);
   }
   if (threadIdx.x == 0) {
      const uint32_t ob = atomicAdd(&counters->dst_top, total);
      s_base = ob;
      if ((uint64_t)ob + total > out_capacity) s_flags |= VLGPU_CELL_NOMEM;
   }
   __syncthreads();
   const bool ok = !(s_flags & VLGPU_CELL_NOMEM);
   const uint32_t obase = s_base;
   if (ok) {
      // emit the new list in global-ID order; data indices default to "added"
      for (uint32_t r = r0; r < r1; ++r) {
         const uint32_t yy = (uint32_t)(y0 + (int)(r % ny)), zz = (uint32_t)(z0 + (int)(r / ny));
         const uint32_t row_gid = L0 * (yy + L1 * zz);
         uint32_t o = obase + prefix[r];
         for (int w = 0; w < 3; ++w) {
            uint32_t m = H[3 * r + w];
            while (m) {
               const int bit = __ffs(m) - 1;
               m &= m - 1;
               out_gids[o] = row_gid + (uint32_t)(w * 32 + bit);
               out_src[o] = NO_BLOCK;
               ++o;
            }
         }
      }
   }
   __syncthreads();
   // old blocks: kept ones point the new entry at their data, removed ones
   // feed the density loss; with the moments fused, the kept blocks' values
   // also give the cell's "_V" moments (MOM_BOTH: the first sums about 0, the
   // second about the pivot's bulk velocity U)
   const bool fuse = mom_record != nullptr;
   double U0 = 0.0, U1 = 0.0, U2 = 0.0;
   if (fuse) {
      const double* pv = pivot + (size_t)cell * MOM_COUNT;
      U0 = pv[MOM_VX]; U1 = pv[MOM_VY]; U2 = pv[MOM_VZ];
   }
   // half a warp per queued block, one x-row of four cells per lane
   const uint32_t half = lane >> 4, sub = lane & 15;
   const double ox = 0.5 * fr.dv[0], oy = ((sub & 3) + 0.5) * fr.dv[1], oz = ((sub >> 2) + 0.5) * fr.dv[2];
   const double dv0s = fr.dv[0] * fr.dv[0];
   double t[10];
#pragma unroll
   for (int q = 0; q < 10; ++q) t[q] = 0.0;
   double lsum = 0.0;  // sum f of the removed blocks (times dv3 below)
   uint32_t* const qidx = s_qidx[warp];
   uint32_t* const qgid = s_qgid[warp];
   const uint32_t lanes_below = (1u << lane) - 1u;
   for (uint32_t b0 = warp * 32; b0 < s.count; b0 += ADJ_THREADS * ADJ_UNROLL) {
      uint32_t qn = 0;
      uint32_t gg[ADJ_UNROLL], ii[ADJ_UNROLL];
#pragma unroll
      for (int u = 0; u < ADJ_UNROLL; ++u) {
         const uint32_t b = b0 + ADJ_THREADS * u + lane;
         gg[u] = b < s.count ? gids[s.off + b] : 0u;
         ii[u] = b < s.count ? (src_index ? src_index[s.off + b] : s.off + b) : NO_BLOCK;
      }
#pragma unroll
      for (int u = 0; u < ADJ_UNROLL; ++u) {
         const bool valid = b0 + ADJ_THREADS * u + lane < s.count;
         uint32_t x, by, bz;
         block_xyz(mesh, gg[u], x, by, bz);
         const int y = (int)by, z = (int)bz;
         bool inH = false;
         uint32_t pos = 0;
         if (valid && any && y >= y0 && y <= y1 && z >= z0 && z <= z1) {
            const uint32_t r = (uint32_t)((z - z0) * ny + (y - y0));
            inH = (H[3 * r + (x >> 5)] >> (x & 31)) & 1u;
            pos = prefix[r] + (uint32_t)mask_popc_below(&H[3 * r], x);
         }
         if (inH && ok) out_src[obase + pos] = ii[u];
         // queue the blocks whose values are read: the removed ones, and with
         // the moments fused the kept ones too
         const bool read = valid && ii[u] != NO_BLOCK && (fuse || !inH);
         const uint32_t bal = __ballot_sync(FULL, read);
         if (read) {
            const uint32_t q = qn + __popc(bal & lanes_below);
            qidx[q] = ii[u];
            qgid[q] = gg[u] | (inH ? ADJ_KEPT : 0u);
         }
         qn += __popc(bal);
      }
      __syncwarp();
      // the queue, eight blocks at a time: half-warp h reads blocks
      // h, h + 2, h + 4, h + 6; the next eight blocks' rows are in flight
      // while these are summed
      auto fetch = [&](uint32_t q0, float4* f, uint32_t* gq) {
#pragma unroll
         for (int v = 0; v < 4; ++v) {
            const uint32_t e = q0 + half + 2 * v;
            gq[v] = e < qn ? qgid[e] : 0xffffffffu;
            f[v] = e < qn ? __ldg(reinterpret_cast<const float4*>(data + (size_t)qidx[e] * WID3) + sub)
                          : make_float4(0.f, 0.f, 0.f, 0.f);
         }
      };
      float4 fc[4], fn[4];
      uint32_t gc[4], gn[4];
      fetch(0, fc, gc);
      for (uint32_t q0 = 0; q0 < qn; q0 += 8) {
         fetch(q0 + 8, fn, gn);
#pragma unroll
         for (int v = 0; v < 4; ++v) {
            if (gc[v] == 0xffffffffu) continue;
            // the row's sums of f, i f and i^2 f (i = 0..3 along x)
            const double d0 = fc[v].x, d1 = fc[v].y, d2 = fc[v].z, d3 = fc[v].w;
            const double s0 = (d0 + d1) + (d2 + d3);
            if (!(gc[v] & ADJ_KEPT)) {
               lsum += s0;
               continue;
            }
            const double s1 = fma(3.0, d3, fma(2.0, d2, d1));
            const double s2 = fma(9.0, d3, fma(4.0, d2, d1));
            uint32_t bi, bj, bk;
            block_xyz(mesh, gc[v] & ~ADJ_KEPT, bi, bj, bk);
            const double x0 = (fr.vmin[0] + bi * fr.bs[0]) + ox;
            const double uy = (fr.vmin[1] + bj * fr.bs[1]) + oy;
            const double uz = (fr.vmin[2] + bk * fr.bs[2]) + oz;
            const double ds1 = fr.dv[0] * s1;
            const double sfx = fma(x0, s0, ds1);  // sum f x over the row
            t[0] += s0;
            t[1] += sfx;
            t[2] = fma(s0, uy, t[2]);
            t[3] = fma(s0, uz, t[3]);
            // the same row relative to U
            const double y0 = x0 - U0, vy = uy - U1, vz = uz - U2;
            const double sfy = fma(y0, s0, ds1);
            t[4] += fma(y0, fma(y0, s0, 2.0 * ds1), dv0s * s2);
            const double s0y = s0 * vy;
            t[5] = fma(s0y, vy, t[5]);
            t[6] = fma(s0 * vz, vz, t[6]);
            t[7] = fma(s0y, vz, t[7]);
            t[8] = fma(sfy, vz, t[8]);
            t[9] = fma(sfy, vy, t[9]);
         }
#pragma unroll
         for (int v = 0; v < 4; ++v) {
            fc[v] = fn[v];
            gc[v] = gn[v];
         }
      }
      __syncwarp();  // the queue is refilled
   }
   // CTA sums of the removed mass and of the moments (fixed order)
#pragma unroll
   for (int o = 16; o >= 1; o >>= 1) lsum += __shfl_xor_sync(FULL, lsum, o);
   if (lane == 0) s_loss[warp] = lsum;
   if (fuse) {
#pragma unroll
      for (int q = 0; q < 10; ++q) {
         double v = t[q];
#pragma unroll
         for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
         if (lane == 0) s_mom[warp][q] = v;
      }
   }
   __syncthreads();
   if (threadIdx.x == 0) {
      double tl = 0.0;
      for (int w = 0; w < ADJ_THREADS / 32; ++w) tl += s_loss[w];
      loss[cell] += dv3 * tl;
      out_slots[cell] = ok ? CellSlot{obase, total} : CellSlot{0u, 0u};
      if (s_flags) atomicOr(&status[cell], s_flags);
      if (!ok) atomicOr(&counters->overflow, 1u);
      if (fuse) {
         double S[10];
         for (int q = 0; q < 10; ++q) {
            double v = 0.0;
            for (int w = 0; w < ADJ_THREADS / 32; ++w) v += s_mom[w][q];
            S[q] = v;
         }
         moments_record<MOM_BOTH>(S, 0.0, 0.0, 0.0, U0, U1, U2, fr.dv[0], fr.dv[1], fr.dv[2], fr.mass, fr.charge,
                                  mom_record + (size_t)cell * MOM_COUNT,
                                  write_pivot ? pivot + (size_t)cell * MOM_COUNT : nullptr);
      }
   }
   __syncthreads();  // the next cell reuses the shared state
   }
}

// Rows of (y, z) masks kept in shared memory; a cell whose box has more uses
// its CTA's global scratch slice.  1600 rows (45 KB) leave room for four CTAs
// per SM.
constexpr uint32_t ADJ_SMEM_ROWS = 1600;
size_t adjust_smem_bytes() { return sizeof(uint32_t) * 7 * ADJ_SMEM_ROWS; }
size_t adjust_scratch_words(const MeshDev& mesh) { return (size_t)7 * mesh.len[1] * mesh.len[2]; }

int adjust_blocks_per_sm() {
   int n = 0;
   cudaFuncSetAttribute(adjust_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)adjust_smem_bytes());
   cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, adjust_kernel, ADJ_THREADS, adjust_smem_bytes());
   return n > 0 ? n : 1;
}

cudaError_t launch_adjust(const uint32_t* gids, const uint32_t* src_index, const CellSlot* slots,
                          const uint8_t* content, const float* data, const int32_t* neighbors, uint32_t* out_gids,
                          uint32_t* out_src,
                          CellSlot* out_slots, double* loss, uint32_t* status, SweepCounters* counters,
                          uint32_t out_capacity, const MeshDev& mesh, double min_value, int add_width, double dv3,
                          uint32_t n_cells, uint32_t* scratch, int grid, const uint32_t* order, MaskRec* masks,
                          uint32_t* pool, uint32_t* pool_top, uint32_t pool_cap, double* mom_record,
                          double* pivot, int write_pivot, const MomentFrame& frame, cudaStream_t stream) {
   if (n_cells == 0) return cudaSuccess;
   const size_t smem = adjust_smem_bytes();
   cudaError_t e = cudaFuncSetAttribute(adjust_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
   if (e != cudaSuccess) return e;
   const bool use_masks = neighbors && masks && pool && pool_top;
   if (use_masks) {
      e = cudaMemsetAsync(pool_top, 0, sizeof(uint32_t), stream);
      if (e != cudaSuccess) return e;
      content_mask_kernel<<<n_cells, MASK_THREADS, 0, stream>>>(gids, src_index, slots, content, data, mesh,
                                                                 min_value, masks, pool, pool_top, pool_cap);
   }
   // the counters' cell_next is zero here (the caller clears the sweep
   // counters before every adjustment)
   const uint32_t g = (uint32_t)grid < n_cells ? (uint32_t)grid : n_cells;
   adjust_kernel<<<g, ADJ_THREADS, smem, stream>>>(gids, src_index, slots, content, data, neighbors, out_gids,
                                                    out_src, out_slots, loss, status, counters, out_capacity, mesh,
                                                    min_value, add_width, dv3, n_cells, ADJ_SMEM_ROWS, scratch,
                                                    use_masks ? masks : nullptr, pool, order, mom_record, pivot,
                                                    write_pivot, frame);
   return cudaGetLastError();
}

}  // namespace vlgpu

namespace vlgpu {

// dst row p = src row src_index[p] (zeros for an added block), p < n_blocks
__global__ void materialize_kernel(const uint32_t* __restrict__ src_index, const float4* __restrict__ src,
                                   float4* __restrict__ dst, uint64_t n_blocks) {
   const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
   const uint64_t p = t >> 4;
   const int q = (int)(t & 15);
   if (p >= n_blocks) return;
   const uint32_t idx = src_index[p];
   dst[p * 16 + q] = (idx == NO_BLOCK) ? make_float4(0.f, 0.f, 0.f, 0.f) : src[(uint64_t)idx * 16 + q];
}

cudaError_t launch_materialize(const uint32_t* src_index, const float* src, float* dst, uint64_t n_blocks,
                               cudaStream_t stream) {
   if (n_blocks == 0) return cudaSuccess;
   const uint64_t threads = n_blocks * 16;
   materialize_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, stream>>>(
      src_index, reinterpret_cast<const float4*>(src), reinterpret_cast<float4*>(dst), n_blocks);
   return cudaGetLastError();
}

// The same for a row count known only on the device (*n_rows), grid-stride.
__global__ void materialize_rows_kernel(const uint32_t* __restrict__ src_index, const float4* __restrict__ src,
                                        float4* __restrict__ dst, const uint32_t* __restrict__ n_rows) {
   const uint64_t n = (uint64_t)(*n_rows) * 16;
   for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
      const uint64_t p = t >> 4;
      const uint32_t idx = src_index[p];
      dst[t] = (idx == NO_BLOCK) ? make_float4(0.f, 0.f, 0.f, 0.f) : src[(uint64_t)idx * 16 + (t & 15)];
   }
}

// Copies the cell slots into mapped pinned host memory: the writes travel as
// a kernel's stores, not through the copy engine, so they do not queue behind
// large device-to-host copies of other streams.
__global__ void slots_to_host_kernel(const CellSlot* __restrict__ src, CellSlot* host_dst, uint32_t n) {
   const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
   if (c < n) host_dst[c] = src[c];
}

cudaError_t launch_slots_to_host(const CellSlot* src, CellSlot* host_dst, uint32_t n, cudaStream_t stream) {
   if (n == 0) return cudaSuccess;
   slots_to_host_kernel<<<(n + 255) / 256, 256, 0, stream>>>(src, host_dst, n);
   return cudaGetLastError();
}

cudaError_t launch_materialize_rows(const uint32_t* src_index, const float* src, float* dst, const uint32_t* n_rows,
                                    int grid, cudaStream_t stream) {
   materialize_rows_kernel<<<grid, 256, 0, stream>>>(src_index, reinterpret_cast<const float4*>(src),
                                                     reinterpret_cast<float4*>(dst), n_rows);
   return cudaGetLastError();
}

}  // namespace vlgpu
