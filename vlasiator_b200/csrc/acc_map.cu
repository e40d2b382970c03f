// SLICE-3D one-dimensional acceleration remap on sparse 4x4x4 velocity blocks
// for sm_100a.  One sweep is two kernels:
//
//   columnize_kernel  one CTA per cell.  Builds the cell's column structure
//                     for the sweep dimension from 96-bit occupancy masks in
//                     shared memory (one mask per transverse block pair),
//                     computes each column's target block range with the
//                     reference's rule (cpu_acc_map.cpp:258-324), allocates
//                     the cell's output blocks and writes one ColumnSet record
//                     per transverse pair plus the source permutation.
//
//   remap_walk_kernel (the default, fused arithmetic) or remap_kernel (the
//                     exact mode): persistent; each half-warp takes one
//                     ColumnSet and walks it along the sweep dimension, one
//                     lane per transverse cell (i,j) of the 4x4 block face.
//                     The reconstruction is built in registers from a sliding
//                     window of the column; each source cell's mass goes to
//                     the Lagrangian target cells it overlaps in a per-lane
//                     ring of 8 target blocks in shared memory, and completed
//                     target blocks are streamed out.  Every output block is
//                     written exactly once, so no zero fill and no atomics are
//                     needed.
//
// remap_kernel follows the reference's scalar build operation by operation
// (round-to-nearest intrinsics, no contraction, the double-precision products
// of cpu_face_estimates.hpp:163 and cpu_acc_map.cpp:585), so its results are
// bit-identical to the reference's map_1d on the same inputs.
#include <cfloat>
#include <cstdint>

#include "fused_ppm.cuh"
#include "vlgpu_common.cuh"

namespace vlgpu {

// ---------------------------------------------------------------------------
// exact IEEE single-precision helpers (never contracted into FMA)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fd(float a, float b) { return __fdiv_rn(a, b); }
// double constant times float, rounded once to float (VecSimple<float> * double)
__device__ __forceinline__ float dmf(double c, float x) { return __double2float_rn(__dmul_rn(c, (double)x)); }

// h4 left face value, cpu_face_estimates.hpp:160-167
__device__ __forceinline__ float h4_face(float vm2, float vm1, float v0, float vp1) {
   float s = fa(-vm2, fm(7.0f, vm1));
   s = fa(s, fm(7.0f, v0));
   s = fs(s, vp1);
   return dmf(1.0 / 12.0, s);
}

__device__ __forceinline__ float minmod(float s1, float s2) {
   const float slope = (fabsf(s1) < fabsf(s2)) ? s1 : s2;
   return (fm(s1, s2) <= 0.0f) ? 0.0f : slope;
}
__device__ __forceinline__ float maxmod(float s1, float s2) {
   const float slope = (fabsf(s1) > fabsf(s2)) ? s1 : s2;
   return (fm(s1, s2) <= 0.0f) ? 0.0f : slope;
}

// PPM coefficients of cpu_1d_ppm.hpp:35-54 (filtered h4 faces, superbee,
// Colella-Woodward monotonicity) for the cell with neighbours vm1, vp1 and
// raw faces fl (left) / fr (right).
__device__ __forceinline__ void ppm_coeff(float vm1, float v0, float vp1, float fl, float fr, float threshold,
                                          float scale, float& a0, float& a1, float& a2) {
   const float l = fm(vm1, scale), m = fm(v0, scale), r = fm(vp1, scale);
   const float a = fs(r, m), b = fs(m, l);
   const float s1 = minmod(a, fm(2.0f, b));
   const float s2 = minmod(fm(2.0f, a), b);
   const float slope = maxmod(s1, s2);
   const float slope_abs = fm(fabsf(slope), threshold);
   const float slope_sign = (slope > 0.0f) ? 1.0f : -1.0f;
   if (slope_abs == 0.0f) {
      fr = v0;
      fl = v0;
   }
   const float half_slope = fm(fm(slope_sign, 0.5f), slope_abs);
   if (fm(fs(vm1, fl), fs(fl, v0)) < 0.0f) fl = fs(v0, half_slope);
   if (fm(fs(vp1, fr), fs(fr, v0)) < 0.0f) fr = fa(v0, half_slope);
   const float one_sixth = (float)(1.0 / 6.0);
   {
      const float d = fs(fr, fl);
      const float e = fs(v0, fm(0.5f, fa(fl, fr)));
      if (fm(d, e) > fm(fm(d, d), one_sixth)) fl = fs(fm(3.0f, v0), fm(2.0f, fr));
   }
   {
      const float d = fs(fr, fl);
      const float e = fs(v0, fm(0.5f, fa(fl, fr)));
      if (fm(fm(-d, d), one_sixth) > fm(d, e)) fr = fs(fm(3.0f, v0), fm(2.0f, fl));
   }
   a0 = fl;
   a1 = fs(fs(fm(3.0f, v0), fm(2.0f, fl)), fr);
   a2 = fs(fa(fl, fr), fm(2.0f, v0));
}

// ---------------------------------------------------------------------------
// 96-bit mask helpers
// ---------------------------------------------------------------------------
// Word q (0..2) of a mask, chosen with selects so that a mask held in
// registers is never indexed dynamically (which would move it to local memory).
__device__ __forceinline__ uint32_t mask_word(const uint32_t m[3], int q) {
   return q == 0 ? m[0] : (q == 1 ? m[1] : m[2]);
}
__device__ __forceinline__ int mask_next_set(const uint32_t m[3], int k) {
   for (; k < 96; k = (k | 31) + 1) {
      const uint32_t w = mask_word(m, k >> 5) >> (k & 31);
      if (w) return k + __ffs(w) - 1;
   }
   return 96;
}
__device__ __forceinline__ int mask_next_clear(const uint32_t m[3], int k) {
   for (; k < 96; k = (k | 31) + 1) {
      const uint32_t w = (~mask_word(m, k >> 5)) >> (k & 31);
      if (w) return k + __ffs(w) - 1;
   }
   return 96;
}

// Target block range of one column (cpu_acc_map.cpp:307-338).  Returns true
// when the range violates the wall margin.
__device__ __forceinline__ bool column_extent(float mx, float mn, float dk, float dv, float v_min, int max_len,
                                              int first_k, int last_k, int wall_margin, int& fb, int& lb) {
   const float first_min_v = fa(fm((float)(WID * first_k), dv), v_min);
   const float last_max_v = fa(fm((float)(WID * (last_k + 1)), dv), v_min);
   const int first_gk = __float2int_rz(fd(fs(first_min_v, mx), dk));
   const int last_gk = __float2int_rz(fd(fs(last_max_v, mn), dk));
   fb = first_gk / WID;
   lb = last_gk / WID;
   fb = (fb >= 0) ? fb : 0;
   fb = (fb < max_len) ? fb : max_len - 1;
   lb = (lb >= 0) ? lb : 0;
   lb = (lb < max_len) ? lb : max_len - 1;
   return fb < wall_margin || fb >= max_len - wall_margin || lb < wall_margin || lb >= max_len - wall_margin;
}

// The set's corner extremes of the Lagrangian starting point
// (cpu_acc_map.cpp:258-288), evaluated exactly as the reference does.
__device__ __forceinline__ void set_corners(const SweepCell& P, uint32_t si, uint32_t sj, float& mx, float& mn) {
   const float A0 = (float)(si * WID), A1 = (float)(si * WID + WID - 1);
   const float B0 = (float)(sj * WID), B1 = (float)(sj * WID + WID - 1);
   const float c00 = fa(fa(P.intersection, fm(A0, P.di)), fm(B0, P.dj));
   const float c01 = fa(fa(P.intersection, fm(A0, P.di)), fm(B1, P.dj));
   const float c10 = fa(fa(P.intersection, fm(A1, P.di)), fm(B0, P.dj));
   const float c11 = fa(fa(P.intersection, fm(A1, P.di)), fm(B1, P.dj));
   mx = c00;
   mx = (mx < c01) ? c01 : mx;
   mx = (mx < c10) ? c10 : mx;
   mx = (mx < c11) ? c11 : mx;
   mn = c00;
   mn = (c01 < mn) ? c01 : mn;
   mn = (c10 < mn) ? c10 : mn;
   mn = (c11 < mn) ? c11 : mn;
}

// ---------------------------------------------------------------------------
// columnize: one CTA per cell
// ---------------------------------------------------------------------------
constexpr int COL_THREADS = 256;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* warp_sums, uint32_t& total) {
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

// The column structure of one cell, by the whole CTA (see the file header).
template <int DIM>
__device__ __forceinline__ void columnize_cell(
   uint32_t cell, const uint32_t* __restrict__ gids, const uint32_t* __restrict__ src_index,
   const CellSlot* __restrict__ src_slots, CellSlot* __restrict__ dst_slots, uint32_t* __restrict__ perm,
   ColumnSet* __restrict__ sets, uint32_t set_capacity, uint32_t dst_capacity,
   const SweepCell* __restrict__ sweep_cells, uint32_t* __restrict__ status, SweepCounters* __restrict__ counters,
   BatchStats* __restrict__ stats, const MeshDev& mesh, int wall_margin, int first_of_step, uint32_t plane_cap,
   uint32_t* __restrict__ wide_cells) {
   extern __shared__ uint32_t smem[];
   __shared__ uint32_t warp_sums[32];
   __shared__ uint32_t s_bbox[4];
   __shared__ uint32_t s_set_base, s_dst_base, s_nsets, s_ntgt, s_flags;

   const CellSlot src = src_slots[cell];
   const SweepCell P = sweep_cells[cell];
   uint32_t li, lj;
   plane_lengths(mesh.len, DIM, li, lj);
   const int max_len = (int)mesh.len[DIM];

   if (threadIdx.x == 0) {
      s_bbox[0] = 0xffffffffu; s_bbox[1] = 0; s_bbox[2] = 0xffffffffu; s_bbox[3] = 0;
      s_flags = 0;
   }
   __syncthreads();
   if (src.count == 0) {
      if (threadIdx.x == 0) dst_slots[cell] = CellSlot{0u, 0u};
      return;
   }
   constexpr uint32_t FULL = 0xffffffffu;
   const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   // pass 1: bounding box of the transverse indices (warp reductions, one
   // shared min/max per warp)
   {
      uint32_t a0 = 0xffffffffu, a1 = 0, b0 = 0xffffffffu, b1 = 0;
      for (uint32_t b = threadIdx.x; b < src.count; b += blockDim.x) {
         uint32_t s[3];
         swapped_indices(gids[src.off + b], mesh.len, DIM, s);
         a0 = min(a0, s[0]); a1 = max(a1, s[0]);
         b0 = min(b0, s[1]); b1 = max(b1, s[1]);
      }
      a0 = __reduce_min_sync(FULL, a0); a1 = __reduce_max_sync(FULL, a1);
      b0 = __reduce_min_sync(FULL, b0); b1 = __reduce_max_sync(FULL, b1);
      if (lane == 0) {
         atomicMin(&s_bbox[0], a0); atomicMax(&s_bbox[1], a1);
         atomicMin(&s_bbox[2], b0); atomicMax(&s_bbox[3], b1);
      }
   }
   __syncthreads();
   const uint32_t a_lo = s_bbox[0], b_lo = s_bbox[2];
   const uint32_t na = s_bbox[1] - a_lo + 1, nb = s_bbox[3] - b_lo + 1;
   const uint32_t plane = na * nb;
   if (plane > plane_cap) {
      // too wide for this launch's shared memory: left to columnize_wide_kernel
      if (threadIdx.x == 0) wide_cells[atomicAdd(&counters->n_wide, 1u)] = cell;
      return;
   }
   uint32_t* mask = smem;                   // 3 * plane
   uint32_t* prefix = smem + 3 * plane;     // plane
   uint16_t* set_t = (uint16_t*)(prefix + plane);  // plane (set index -> t)
   uint32_t* tcount = prefix + plane + (plane + 1) / 2;  // plane
   for (uint32_t q = threadIdx.x; q < 3 * plane; q += blockDim.x) mask[q] = 0;
   __syncthreads();
   // pass 2: occupancy masks along the sweep dimension; lanes that set bits
   // of one word (a run of the list along the sweep) combine them first
   for (uint32_t b0 = warp * 32; b0 < src.count; b0 += blockDim.x) {
      const uint32_t b = b0 + lane;
      uint32_t key = 0xffffffffu, bit = 0u;
      if (b < src.count) {
         uint32_t s[3];
         swapped_indices(gids[src.off + b], mesh.len, DIM, s);
         key = 3 * ((s[0] - a_lo) * nb + (s[1] - b_lo)) + (s[2] >> 5);
         bit = 1u << (s[2] & 31);
      }
      const uint32_t match = __match_any_sync(FULL, key);
      const bool big = key != 0xffffffffu && __popc(match) >= 4;
      if (key != 0xffffffffu && !big) atomicOr(&mask[key], bit);
      for (uint32_t leaders = __ballot_sync(FULL, big && (int)lane == __ffs(match) - 1); leaders;
           leaders &= leaders - 1) {
         const int leader = __ffs(leaders) - 1;
         const bool mine = (__shfl_sync(FULL, match, leader) >> lane) & 1u;
         const uint32_t bits = __reduce_or_sync(FULL, mine ? bit : 0u);
         if ((int)lane == leader) atomicOr(&mask[key], bits);
      }
   }
   __syncthreads();
   // scan over the plane: source offsets and set indices
   const uint32_t chunk = (plane + blockDim.x - 1) / blockDim.x;
   const uint32_t t0 = min(plane, threadIdx.x * chunk), t1 = min(plane, t0 + chunk);
   uint32_t my_blocks = 0, my_sets = 0;
   for (uint32_t t = t0; t < t1; ++t) {
      const uint32_t n = __popc(mask[3 * t]) + __popc(mask[3 * t + 1]) + __popc(mask[3 * t + 2]);
      my_blocks += n;
      my_sets += (n > 0);
   }
   uint32_t tot_blocks, tot_sets;
   uint32_t blk_base = block_exclusive_scan(my_blocks, warp_sums, tot_blocks);
   uint32_t set_base = block_exclusive_scan(my_sets, warp_sums, tot_sets);
   for (uint32_t t = t0; t < t1; ++t) {
      const uint32_t n = __popc(mask[3 * t]) + __popc(mask[3 * t + 1]) + __popc(mask[3 * t + 2]);
      prefix[t] = blk_base;
      blk_base += n;
      if (n > 0) set_t[set_base++] = (uint16_t)t;
   }
   if (threadIdx.x == 0) {
      const uint32_t base = atomicAdd(&counters->n_sets, tot_sets);
      s_set_base = base;
      s_nsets = tot_sets;
      if (base + tot_sets > set_capacity) s_flags |= VLGPU_CELL_NOMEM;
   }
   __syncthreads();
   const bool sets_ok = !(s_flags & VLGPU_CELL_NOMEM);
   // per set: target mask from the column extents
   uint32_t wall = 0, baddk = 0;
   for (uint32_t s = threadIdx.x; s < tot_sets; s += blockDim.x) {
      const uint32_t t = set_t[s];
      const uint32_t si = a_lo + t / nb, sj = b_lo + t % nb;
      uint32_t m[3] = {mask[3 * t], mask[3 * t + 1], mask[3 * t + 2]};
      uint32_t tm[3] = {0u, 0u, 0u};
      if (P.flags & SWEEP_PASS) {
         // the cell's blocks pass through the sweep unchanged
         tm[0] = m[0]; tm[1] = m[1]; tm[2] = m[2];
      } else {
         float mx, mn;
         set_corners(P, si, sj, mx, mn);
         if (!(P.dk > 0.0f)) baddk = 1;
         int k = mask_next_set(m, 0);
         while (k < 96) {
            const int e = mask_next_clear(m, k) - 1;
            int fb, lb;
            if (column_extent(mx, mn, P.dk, mesh.dv[DIM], mesh.vmin[DIM], max_len, k, e, wall_margin, fb, lb))
               wall = 1;
            for (int q = fb; q <= lb; ++q) tm[q >> 5] |= 1u << (q & 31);
            k = mask_next_set(m, e + 1);
         }
      }
      tcount[s] = __popc(tm[0]) + __popc(tm[1]) + __popc(tm[2]);
      if (sets_ok) {
         ColumnSet cs;
         cs.cell = cell;
         cs.si = si;
         cs.sj = sj;
         cs.src_pos = src.off + prefix[t];
         cs.dst_pos = 0;
         cs.src_mask[0] = m[0]; cs.src_mask[1] = m[1]; cs.src_mask[2] = m[2];
         cs.tgt_mask[0] = tm[0]; cs.tgt_mask[1] = tm[1]; cs.tgt_mask[2] = tm[2];
         sets[s_set_base + s] = cs;
      }
   }
   if (wall) atomicOr(&s_flags, VLGPU_CELL_WALL);
   if (baddk) atomicOr(&s_flags, VLGPU_CELL_BADDK);
   __syncthreads();
   // scan of target counts over sets -> output positions
   const uint32_t sch = (tot_sets + blockDim.x - 1) / blockDim.x;
   const uint32_t q0 = min(tot_sets, threadIdx.x * sch), q1 = min(tot_sets, q0 + sch);
   uint32_t my_t = 0;
   for (uint32_t s = q0; s < q1; ++s) my_t += tcount[s];
   uint32_t tot_t;
   uint32_t tbase = block_exclusive_scan(my_t, warp_sums, tot_t);
   if (threadIdx.x == 0) {
      const uint32_t base = atomicAdd(&counters->dst_top, tot_t);
      s_dst_base = base;
      s_ntgt = tot_t;
      if ((uint64_t)base + tot_t > dst_capacity) s_flags |= VLGPU_CELL_NOMEM;
   }
   __syncthreads();
   const bool ok = !(s_flags & VLGPU_CELL_NOMEM);
   if (ok) {
      for (uint32_t s = q0; s < q1; ++s) {
         sets[s_set_base + s].dst_pos = s_dst_base + tbase;
         tbase += tcount[s];
      }
      // source permutation in (set, k) order
      for (uint32_t b = threadIdx.x; b < src.count; b += blockDim.x) {
         uint32_t s[3];
         swapped_indices(gids[src.off + b], mesh.len, DIM, s);
         const uint32_t t = (s[0] - a_lo) * nb + (s[1] - b_lo);
         const uint32_t pos = prefix[t] + (uint32_t)mask_popc_below(&mask[3 * t], s[2]);
         perm[src.off + pos] = src_index ? src_index[src.off + b] : src.off + b;
      }
   } else if (sets_ok) {
      // no room for the output: neutralise this cell's sets
      for (uint32_t s = threadIdx.x; s < tot_sets; s += blockDim.x) {
         sets[s_set_base + s].tgt_mask[0] = 0;
         sets[s_set_base + s].tgt_mask[1] = 0;
         sets[s_set_base + s].tgt_mask[2] = 0;
         sets[s_set_base + s].src_mask[0] = 0;
         sets[s_set_base + s].src_mask[1] = 0;
         sets[s_set_base + s].src_mask[2] = 0;
      }
   }
   if (threadIdx.x == 0) {
      atomicAdd(&stats->src_blocks, (unsigned long long)src.count);
      atomicAdd(&stats->dst_blocks, (unsigned long long)(ok ? s_ntgt : 0u));
      atomicAdd(&stats->sweeps, 1ull);
      atomicAdd(&stats->sets, (unsigned long long)tot_sets);
      if (first_of_step) atomicAdd(&stats->step_blocks, (unsigned long long)src.count);
      dst_slots[cell] = ok ? CellSlot{s_dst_base, s_ntgt} : CellSlot{0u, 0u};
      if (s_flags) atomicOr(&status[cell], s_flags);
      if (!ok) atomicOr(&counters->overflow, 1u);
   }
}

// One CTA per cell of [cell_begin, cell_end).
template <int DIM>
__global__ void __launch_bounds__(COL_THREADS) columnize_kernel(
   const uint32_t* __restrict__ gids, const uint32_t* __restrict__ src_index, const CellSlot* __restrict__ src_slots,
   CellSlot* __restrict__ dst_slots, uint32_t* __restrict__ perm, ColumnSet* __restrict__ sets,
   uint32_t set_capacity, uint32_t dst_capacity,
   const SweepCell* __restrict__ sweep_cells, uint32_t* __restrict__ status, SweepCounters* __restrict__ counters,
   BatchStats* __restrict__ stats, MeshDev mesh, int wall_margin, uint32_t cell_begin, uint32_t cell_end,
   int first_of_step, const uint32_t* __restrict__ order, uint32_t plane_cap, uint32_t* __restrict__ wide_cells) {
   if (cell_begin + blockIdx.x >= cell_end) return;
   const uint32_t cell = order ? order[blockIdx.x] : cell_begin + blockIdx.x;
   columnize_cell<DIM>(cell, gids, src_index, src_slots, dst_slots, perm, sets, set_capacity, dst_capacity,
                       sweep_cells, status, counters, stats, mesh, wall_margin, first_of_step, plane_cap,
                       wide_cells);
}

// Persistent CTAs over the cells whose plane did not fit the capped launch
// (wide_cells, counters->n_wide of them), with a full plane of shared memory.
template <int DIM>
__global__ void __launch_bounds__(COL_THREADS) columnize_wide_kernel(
   const uint32_t* __restrict__ gids, const uint32_t* __restrict__ src_index, const CellSlot* __restrict__ src_slots,
   CellSlot* __restrict__ dst_slots, uint32_t* __restrict__ perm, ColumnSet* __restrict__ sets,
   uint32_t set_capacity, uint32_t dst_capacity,
   const SweepCell* __restrict__ sweep_cells, uint32_t* __restrict__ status, SweepCounters* __restrict__ counters,
   BatchStats* __restrict__ stats, MeshDev mesh, int wall_margin, int first_of_step,
   const uint32_t* __restrict__ wide_cells) {
   const uint32_t n = counters->n_wide;
   for (uint32_t it = blockIdx.x; it < n; it += gridDim.x) {
      columnize_cell<DIM>(wide_cells[it], gids, src_index, src_slots, dst_slots, perm, sets, set_capacity,
                          dst_capacity, sweep_cells, status, counters, stats, mesh, wall_margin, first_of_step,
                          0xffffffffu, nullptr);
      __syncthreads();  // the next cell reuses the shared state
   }
}

// Dynamic shared memory of columnize for a full transverse plane.
size_t columnize_smem_bytes(uint32_t plane) {
   return sizeof(uint32_t) * (3 * plane + plane + (plane + 1) / 2 + plane) + 16;
}

// ---------------------------------------------------------------------------
// remap: persistent, one half-warp per column set
// ---------------------------------------------------------------------------
constexpr int REMAP_THREADS = 256;
constexpr int RING_BLOCKS = 8;               // target blocks held per set
constexpr int RING_CELLS = RING_BLOCKS * WID;  // per lane
constexpr int RING_STRIDE = RING_CELLS * 16 + 16;  // floats per half-warp (+16 pad: bank shift)
// remap_walk_kernel keeps each lane's ring contiguous: 32 cells padded to 36
// floats, so a block's four cells are one aligned 16-byte access (lanes that
// store to the same slot share 8 bank groups, a conflict the measured kernel
// pays for less than it saves in flush instructions)
constexpr int WALK_LANE_STRIDE = RING_CELLS + 4;

template <int DIM>
__device__ __forceinline__ int cell_offset(int i, int j, int g) {
   if (DIM == 0) return i * WID2 + j * WID + g;
   if (DIM == 1) return i + j * WID2 + g * WID;
   return i + j * WID + g * WID2;
}

constexpr uint32_t NO_BLOCK = 0xffffffffu;  // a block that exists with all-zero data

__device__ __forceinline__ int clampi(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }

template <int DIM>
__device__ __forceinline__ void load_lane(const float* __restrict__ data, uint32_t idx, int i, int j, float v[4]) {
   if (idx == NO_BLOCK) {
      v[0] = v[1] = v[2] = v[3] = 0.0f;
      return;
   }
   const float* __restrict__ blk = data + (size_t)idx * WID3;
   if (DIM == 0) {
      const float4 q = __ldg(reinterpret_cast<const float4*>(blk + cell_offset<0>(i, j, 0)));
      v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
   } else {
#pragma unroll
      for (int g = 0; g < 4; ++g) v[g] = __ldg(blk + cell_offset<DIM>(i, j, g));
   }
}

template <int DIM>
__device__ __forceinline__ void store_lane(float* __restrict__ blk, int i, int j, const float v[4]) {
   if (DIM == 0) {
      *reinterpret_cast<float4*>(blk + cell_offset<0>(i, j, 0)) = make_float4(v[0], v[1], v[2], v[3]);
   } else {
#pragma unroll
      for (int g = 0; g < 4; ++g) blk[cell_offset<DIM>(i, j, g)] = v[g];
   }
}

// The set of a cell that is not accelerated in this step (SWEEP_PASS): its
// blocks are copied to the output in ascending k, which is the target mask's
// order (columnize gave the set its source mask as the target mask), with
// their block IDs and content flags.
template <int DIM>
__device__ __forceinline__ void pass_through_set(const ColumnSet& cs, const uint32_t* __restrict__ perm,
                                                 const float* __restrict__ src_data, float* __restrict__ dst_data,
                                                 uint32_t* __restrict__ dst_gids, uint8_t* __restrict__ content_out,
                                                 const MeshDev& mesh, float content_thr, int lane, unsigned hmask) {
   const int i = lane & 3, j = lane >> 2;
   uint32_t r = 0;
   for (int k = mask_next_set(cs.src_mask, 0); k < 96; k = mask_next_set(cs.src_mask, k + 1), ++r) {
      float v[4];
      load_lane<DIM>(src_data, perm[cs.src_pos + r], i, j, v);
      const uint32_t o = cs.dst_pos + r;
      store_lane<DIM>(dst_data + (size_t)o * WID3, i, j, v);
      const bool c = fmaxf(fmaxf(v[0], v[1]), fmaxf(v[2], v[3])) >= content_thr;
      const unsigned any_c = __ballot_sync(hmask, c) & hmask;
      if (lane == 0) {
         dst_gids[o] = gid_from_swapped(cs.si, cs.sj, (uint32_t)k, mesh.len, DIM);
         content_out[o] = any_c ? 1 : 0;
      }
   }
}

// Reference argmax / argmin lane selection (cpu_acc_map.cpp:515-529): the
// first lane holding the largest value above DBL_MIN (default lane 0) and the
// first lane holding the smallest value below DBL_MAX (default lane 0).
__device__ __forceinline__ void select_lanes(float lag, int lane, unsigned hmask, int& max_lane, int& min_lane) {
   bool vmax = (double)lag > DBL_MIN;
   float xmax = lag;
   int imax = lane;
   bool vmin = (double)lag < DBL_MAX;
   float xmin = lag;
   int imin = lane;
#pragma unroll
   for (int o = 8; o >= 1; o >>= 1) {
      const bool ov = __shfl_xor_sync(hmask, vmax, o, 16);
      const float ox = __shfl_xor_sync(hmask, xmax, o, 16);
      const int oi = __shfl_xor_sync(hmask, imax, o, 16);
      if (ov && (!vmax || ox > xmax || (ox == xmax && oi < imax))) { vmax = true; xmax = ox; imax = oi; }
      const bool nv = __shfl_xor_sync(hmask, vmin, o, 16);
      const float nx = __shfl_xor_sync(hmask, xmin, o, 16);
      const int ni = __shfl_xor_sync(hmask, imin, o, 16);
      if (nv && (!vmin || nx < xmin || (nx == xmin && ni < imin))) { vmin = true; xmin = nx; imin = ni; }
   }
   max_lane = vmax ? imax : 0;
   min_lane = vmin ? imin : 0;
}

template <int DIM>
__global__ void __launch_bounds__(REMAP_THREADS, 3) remap_kernel(
   const ColumnSet* __restrict__ sets, SweepCounters* __restrict__ counters, const uint32_t* __restrict__ perm,
   const float* __restrict__ src_data, float* __restrict__ dst_data, uint32_t* __restrict__ dst_gids,
   const SweepCell* __restrict__ sweep_cells, uint32_t* __restrict__ status, MeshDev mesh, int wall_margin,
   uint32_t set_capacity, uint8_t* __restrict__ content_out, double content_threshold) {
   __shared__ float ring_all[(REMAP_THREADS / 16) * RING_STRIDE];
   const int hw = threadIdx.x >> 4;
   const int lane = threadIdx.x & 15;
   const unsigned hmask = 0xffffu << (threadIdx.x & 16);
   float* ring = ring_all + hw * RING_STRIDE;
   const int i = lane & 3, j = lane >> 2;
   uint32_t n_sets = *((volatile uint32_t*)&counters->n_sets);
   n_sets = (n_sets < set_capacity) ? n_sets : set_capacity;
   const int max_len = (int)mesh.len[DIM];
   const float dv = mesh.dv[DIM], v_min = mesh.vmin[DIM];
   const double i_dv = 1.0 / (double)dv;
   // (double)v >= content_threshold  <=>  v >= the smallest float >= the threshold
   const float content_thr = __double2float_ru(content_threshold);

   // the ring starts empty; every set flushes all its targets, and a flush
   // zeroes the slots it reads, so the ring is empty again at each set start
#pragma unroll
   for (int q = 0; q < RING_CELLS; ++q) ring[q * 16 + lane] = 0.0f;
   for (;;) {
      uint32_t sidx = 0;
      if (lane == 0) sidx = atomicAdd(&counters->work, 1u);
      sidx = __shfl_sync(hmask, sidx, 0, 16);
      if (sidx >= n_sets) break;
      const ColumnSet cs = sets[sidx];
      const SweepCell P = sweep_cells[cs.cell];
      if (P.flags & SWEEP_PASS) {
         pass_through_set<DIM>(cs, perm, src_data, dst_data, dst_gids, content_out, mesh, content_thr, lane, hmask);
         continue;
      }
      const float threshold = P.threshold;
      const float scale = __double2float_rn(1.0 / (double)threshold);
      const float dk = P.dk;
      // lane's Lagrangian starting point (cpu_acc_map.cpp:493-496)
      const float A = fa((float)(cs.si * WID), (float)i);
      const float B = fa((float)(cs.sj * WID), (float)j);
      const float im = fa(fa(P.intersection, fm(A, P.di)), fm(B, P.dj));
      float mx, mn;
      set_corners(P, cs.si, cs.sj, mx, mn);
      int next_flush = mask_next_set(cs.tgt_mask, 0);
      uint32_t out_idx = 0;
      bool range_err = false;

      // writes out every target block below `limit_block` that is still held
      auto flush_until = [&](int limit_block) {
         while (next_flush < 96 && next_flush < limit_block) {
            float v[4];
            const int slot = (next_flush & (RING_BLOCKS - 1)) * WID;
#pragma unroll
            for (int g = 0; g < 4; ++g) {
               v[g] = ring[(slot + g) * 16 + lane];
               ring[(slot + g) * 16 + lane] = 0.0f;
            }
            const uint32_t o = cs.dst_pos + out_idx;
            store_lane<DIM>(dst_data + (size_t)o * WID3, i, j, v);
            // content flag of the finished block (compute_block_has_content)
            const bool c = (v[0] >= content_thr) | (v[1] >= content_thr) | (v[2] >= content_thr) |
                           (v[3] >= content_thr);
            const unsigned any_c = __ballot_sync(hmask, c) & hmask;
            if (lane == 0) {
               dst_gids[o] = gid_from_swapped(cs.si, cs.sj, (uint32_t)next_flush, mesh.len, DIM);
               content_out[o] = any_c ? 1 : 0;
            }
            ++out_idx;
            next_flush = mask_next_set(cs.tgt_mask, next_flush + 1);
         }
      };

      int src_rank = 0;
      int col_s = mask_next_set(cs.src_mask, 0);
      int col_e = (col_s < 96) ? mask_next_clear(cs.src_mask, col_s) - 1 : 95;
      int cf = 0, cl = 0;
      if (col_s < 96) column_extent(mx, mn, dk, dv, v_min, max_len, col_s, col_e, wall_margin, cf, cl);
      while (col_s < 96) {
         const int nxt_s = mask_next_set(cs.src_mask, col_e + 1);
         int nxt_e = 95, ncf = 1 << 20, ncl = 0;
         if (nxt_s < 96) {
            nxt_e = mask_next_clear(cs.src_mask, nxt_s) - 1;
            column_extent(mx, mn, dk, dv, v_min, max_len, nxt_s, nxt_e, wall_margin, ncf, ncl);
         }
         // ---- map one column (cpu_acc_map.cpp:395-631) ----
         float v_r = fa(fm((float)(WID * col_s), dv), v_min);
         int gk_r;
         int max_lane = 0, min_lane = 0;
         {
            const float lag = fd(fs(v_r, im), dk);
            gk_r = __float2int_rz(lag);
            select_lanes(lag, lane, hmask, max_lane, min_lane);
         }
         const int gk_lo_col = cf * WID, gk_hi_col = (cl + 1) * WID - 1;
         float pw[4] = {0.0f, 0.0f, 0.0f, 0.0f};  // the previous block (zero padding at a column start)
         float cur[4], nxt[4];
         load_lane<DIM>(src_data, perm[cs.src_pos + src_rank], i, j, cur);
         if (col_e > col_s) {
            load_lane<DIM>(src_data, perm[cs.src_pos + src_rank + 1], i, j, nxt);
         } else {
            nxt[0] = nxt[1] = nxt[2] = nxt[3] = 0.0f;
         }
         // raw left face of the column's first cell
         float face = h4_face(pw[2], pw[3], cur[0], cur[1]);
         for (int kb = col_s; kb <= col_e; ++kb) {
            float nn[4];
            if (kb + 2 <= col_e) {
               load_lane<DIM>(src_data, perm[cs.src_pos + src_rank + 2], i, j, nn);
            } else {
               nn[0] = nn[1] = nn[2] = nn[3] = 0.0f;
            }
            // cell g of the block is w[g + 4]; the stencil reaches 2 cells each way
            const float w[12] = {pw[0], pw[1], pw[2], pw[3], cur[0], cur[1], cur[2], cur[3],
                                 nxt[0], nxt[1], nxt[2], nxt[3]};
#pragma unroll
            for (int g = 0; g < 4; ++g) {
               float a[3];
               const float fr = h4_face(w[g + 3], w[g + 4], w[g + 5], w[g + 6]);
               ppm_coeff(w[g + 3], w[g + 4], w[g + 5], face, fr, threshold, scale, a[0], a[1], a[2]);
               face = fr;
               const float v_l = v_r;
               v_r = fa(v_r, dv);
               const int gk_l = gk_r;
               gk_r = __float2int_rz(fd(fs(v_r, im), dk));
               int min_gk = __shfl_sync(hmask, gk_l, min_lane, 16);
               int max_gk = __shfl_sync(hmask, gk_r, max_lane, 16);
               min_gk = (min_gk > gk_lo_col) ? min_gk : gk_lo_col;
               max_gk = (max_gk < gk_hi_col) ? max_gk : gk_hi_col;
               if (max_gk >= min_gk) {
                  if ((min_gk >> 2) < next_flush || (max_gk >> 2) >= next_flush + RING_BLOCKS) {
                     range_err = true;
                  } else {
                     float dens_r = 0.0f;
                     for (int gk = min_gk; gk <= max_gk; ++gk) {
                        float x = fa(fm((float)(gk + 1), dk), im);
                        x = (x > v_l) ? x : v_l;
                        x = (x < v_r) ? x : v_r;
                        const float u = __double2float_rn(__dmul_rn((double)fs(x, v_l), i_dv));
                        const float dl = dens_r;
                        dens_r = fm(u, fa(a[0], fm(u, fa(a[1], fm(u, a[2])))));
                        float* t = &ring[(gk & (RING_CELLS - 1)) * 16 + lane];
                        *t = fa(*t, fs(dens_r, dl));
                     }
                  }
               }
            }
            // targets below the next source cell's lower bound are complete
            int lb = ncf * WID;
            if (kb < col_e) {
               int nl = __shfl_sync(hmask, gk_r, min_lane, 16);
               nl = (nl > gk_lo_col) ? nl : gk_lo_col;
               lb = (nl < lb) ? nl : lb;
            }
            flush_until(lb >> 2);
#pragma unroll
            for (int g = 0; g < 4; ++g) {
               pw[g] = cur[g];
               cur[g] = nxt[g];
               nxt[g] = nn[g];
            }
            ++src_rank;
         }
         col_s = nxt_s;
         col_e = nxt_e;
         cf = ncf;
         cl = ncl;
      }
      flush_until(1 << 20);
      if (__any_sync(hmask, range_err)) {
         if (lane == 0) atomicOr(&status[cs.cell], VLGPU_CELL_RANGE);
         // deposits past the ring window may have landed in slots no flush
         // reads: clear the ring so that the next set starts empty
#pragma unroll
         for (int q = 0; q < RING_CELLS; ++q) ring[q * 16 + lane] = 0.0f;
      }
   }
}

// ---------------------------------------------------------------------------
// remap_walk: the fused arithmetic as a single-accumulator walk
// ---------------------------------------------------------------------------
// The same column sets, lanes, ring and flushes as remap_kernel, with the
// reconstruction and the distribution of mass over the target cells reduced
// to what the fused mode needs:
//
//  - PPM: each face's raw h4 value and its test "face outside the values of
//    the two cells it separates" are evaluated once and used by both cells
//    (the test of the left face of cell k, (v_{k-1} - f)(f - v_k) < 0, is the
//    test of the right face of cell k-1 with the same rounded product); the two
//    Colella-Woodward overshoot corrections are applied as alternatives (in
//    exact arithmetic the second can no longer fire once the first has).
//  - Distribution: each lane keeps one pending target g (the lowest target
//    cell not yet complete), its accumulated mass and the position u of the
//    target's right edge (g+1) dk + im relative to the current source cell,
//    in units of dv.  A source cell with the edge inside (u < 1) completes
//    target g with the integral up to the edge and starts target g+1 with the
//    rest of the cell (v0 - D(u), so the cell's mass is kept exactly as a
//    sum); otherwise the whole cell goes to target g.  A second edge inside
//    one source cell (dk < dv) takes a rare loop.
//  - Ring traffic: a completed target is stored once into the lane's ring
//    slot.  Within a column a lane completes each target cell once, and the
//    targets of different columns of a set never share a cell while dk < 4 dv
//    (a target would have to span the empty block between them); the first
//    target of a column starts from what its slot already holds (the last
//    target of the column before it, when dk >= 4 dv), so targets shared by
//    two columns are summed in every case.  A flush zeroes the slots it reads.
//  - Target limits of the column (cpu_acc_map.cpp:559-569): a lane whose first
//    target lies below the column's lowest target cell starts at that cell,
//    which then receives all mass below its right edge, as in the reference;
//    mass of targets above the column's highest cell is moved into it when
//    the column ends.
template <int DIM, int RECON>
__global__ void __launch_bounds__(REMAP_THREADS, RECON == RECON_PQM ? 2 : 4) remap_walk_kernel(
   const ColumnSet* __restrict__ sets, SweepCounters* __restrict__ counters, const uint32_t* __restrict__ perm,
   const float* __restrict__ src_data, float* __restrict__ dst_data, uint32_t* __restrict__ dst_gids,
   const SweepCell* __restrict__ sweep_cells, uint32_t* __restrict__ status, MeshDev mesh, int wall_margin,
   uint32_t set_capacity, uint8_t* __restrict__ content_out, double content_threshold) {
   __shared__ __align__(16) float ring_all[REMAP_THREADS * WALK_LANE_STRIDE];
   const int hw = threadIdx.x >> 4;
   const int lane = threadIdx.x & 15;
   const unsigned hmask = 0xffffu << (threadIdx.x & 16);
   // this lane's slots ring[t], t = target cell mod RING_CELLS, contiguous so
   // that a target block's four cells are one 16-byte access
   float* ring = ring_all + (size_t)threadIdx.x * WALK_LANE_STRIDE;
   const int i = lane & 3, j = lane >> 2;
   uint32_t n_sets = *((volatile uint32_t*)&counters->n_sets);
   n_sets = (n_sets < set_capacity) ? n_sets : set_capacity;
   const int max_len = (int)mesh.len[DIM];
   const float dv = mesh.dv[DIM], v_min = mesh.vmin[DIM];
   const float inv_dv = (float)(1.0 / (double)dv);
   const float content_thr = __double2float_ru(content_threshold);
   constexpr float one_sixth = (float)(1.0 / 6.0);
   constexpr int RMASK = RING_CELLS - 1;
   constexpr uint32_t SMASK = RING_CELLS - 1;  // slot offsets wrap around the ring

#pragma unroll
   for (int q = 0; q < RING_CELLS; ++q) ring[q] = 0.0f;
   for (;;) {
      uint32_t sidx = 0;
      if (lane == 0) sidx = atomicAdd(&counters->work, 1u);
      sidx = __shfl_sync(hmask, sidx, 0, 16);
      if (sidx >= n_sets) break;
      const ColumnSet cs = sets[sidx];
      const SweepCell P = sweep_cells[cs.cell];
      if (P.flags & SWEEP_PASS) {
         pass_through_set<DIM>(cs, perm, src_data, dst_data, dst_gids, content_out, mesh, content_thr, lane, hmask);
         continue;
      }
      const float dk = P.dk;
      const float A = fa((float)(cs.si * WID), (float)i);
      const float B = fa((float)(cs.sj * WID), (float)j);
      const float im = fa(fa(P.intersection, fm(A, P.di)), fm(B, P.dj));
      float mx, mn;
      set_corners(P, cs.si, cs.sj, mx, mn);
      const uint32_t gid0 = gid_from_swapped(cs.si, cs.sj, 0u, mesh.len, DIM);
      const uint32_t gid_step = gid_from_swapped(cs.si, cs.sj, 1u, mesh.len, DIM) - gid0;
      // the next target block to write and the end of the run of consecutive
      // target blocks it belongs to
      int next_flush = mask_next_set(cs.tgt_mask, 0);
      int run_end = mask_next_clear(cs.tgt_mask, next_flush);
      uint32_t out_idx = 0;
      bool range_err = false;

      auto flush_until = [&](int limit_block) {
         while (next_flush < 96 && next_flush < limit_block) {
            const int slot = (next_flush & (RING_BLOCKS - 1)) * WID;
            const float4 v4 = *reinterpret_cast<const float4*>(ring + slot);
            *reinterpret_cast<float4*>(ring + slot) = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            const float v[4] = {v4.x, v4.y, v4.z, v4.w};
            const uint32_t o = cs.dst_pos + out_idx;
            store_lane<DIM>(dst_data + (size_t)o * WID3, i, j, v);
            const bool c = fmaxf(fmaxf(v[0], v[1]), fmaxf(v[2], v[3])) >= content_thr;
            const unsigned any_c = __ballot_sync(hmask, c) & hmask;
            if (lane == 0) {
               dst_gids[o] = gid0 + (uint32_t)next_flush * gid_step;
               content_out[o] = any_c ? 1 : 0;
            }
            ++out_idx;
            if (++next_flush >= run_end) {
               next_flush = mask_next_set(cs.tgt_mask, next_flush);
               run_end = mask_next_clear(cs.tgt_mask, next_flush);
            }
         }
      };

      // a cell whose Lagrangian cells do not advance (flagged by columnize)
      // gets its target blocks with zero values
      const bool walkable = dk > 0.0f;
      int src_rank = 0;
      int col_s = walkable ? mask_next_set(cs.src_mask, 0) : 96;
      int col_e = (col_s < 96) ? mask_next_clear(cs.src_mask, col_s) - 1 : 95;
      int cf = 0, cl = 0;
      if (col_s < 96) column_extent(mx, mn, dk, dv, v_min, max_len, col_s, col_e, wall_margin, cf, cl);
      while (col_s < 96) {
         const int nxt_s = mask_next_set(cs.src_mask, col_e + 1);
         int nxt_e = 95, ncf = 1 << 20, ncl = 0;
         if (nxt_s < 96) {
            nxt_e = mask_next_clear(cs.src_mask, nxt_s) - 1;
            column_extent(mx, mn, dk, dv, v_min, max_len, nxt_s, nxt_e, wall_margin, ncf, ncl);
         }
         const int lo = cf * WID, hi = (cl + 1) * WID - 1;
         // ---- the lane's first target: the lowest g with (g+1) dk + im > v_l ----
         float v_l = fa(fm((float)(WID * col_s), dv), v_min);
         int g = __float2int_rz(fd(fs(v_l, im), dk));
         float e = fa(fm((float)(g + 1), dk), im);
         for (int q = 0; q < 3 && e <= v_l; ++q) {
            ++g;
            e = fa(fm((float)(g + 1), dk), im);
         }
         for (int q = 0; q < 3; ++q) {
            const float ep = fa(fm((float)g, dk), im);
            if (!(ep > v_l)) break;
            --g;
            e = ep;
         }
         if (g < lo) {
            g = lo;
            e = fa(fm((float)(g + 1), dk), im);
         }
         float g1f = (float)(g + 1);   // the pending target's edge index (g + 1)
         uint32_t soff = (uint32_t)(g & RMASK);  // the pending target's slot
         float u = fs(e, v_l) * inv_dv;
         // minus the pending target's accumulated mass (kept negated so that
         // both branches of the per-cell update are one select and one add)
         float nacc = -ring[soff];  // what another column left in the slot
         float pw0 = 0.0f, pw1 = 0.0f, pw2 = 0.0f, pw3 = 0.0f;  // cells below the block (zero padding)
         float cur[4], nxt[4];
         load_lane<DIM>(src_data, perm[cs.src_pos + src_rank], i, j, cur);
         if (col_e > col_s) {
            load_lane<DIM>(src_data, perm[cs.src_pos + src_rank + 1], i, j, nxt);
         } else {
            nxt[0] = nxt[1] = nxt[2] = nxt[3] = 0.0f;
         }
         // face state of the column's first cell
         float face = 0.0f, face_d = 0.0f;
         bool face_out = false;  // PPM: the left face lies outside its two cells' values
         float dprev = cur[0];   // v_k - v_{k-1}
         if constexpr (RECON == RECON_PPM) {
            face = h4_face_fused(0.0f, 0.0f, cur[0], cur[1]);
            face_out = (0.0f - face) * (face - cur[0]) < 0.0f;
         }
         if constexpr (RECON == RECON_PQM) {
            face = h8_value(0.0f, 0.0f, 0.0f, 0.0f, cur[0], cur[1], cur[2], cur[3]);
            face_d = h7_derivative(0.0f, 0.0f, 0.0f, 0.0f, cur[0], cur[1], cur[2], cur[3]);
         }
         for (int kb = col_s; kb <= col_e; ++kb) {
            float nn[4];
            if (kb + 2 <= col_e) {
               load_lane<DIM>(src_data, perm[cs.src_pos + src_rank + 2], i, j, nn);
            } else {
               nn[0] = nn[1] = nn[2] = nn[3] = 0.0f;
            }
            const float w[12] = {pw0, pw1, pw2, pw3, cur[0], cur[1], cur[2], cur[3], nxt[0], nxt[1], nxt[2], nxt[3]};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
               const float vm1 = w[q + 3], v0 = w[q + 4], vp1 = w[q + 5];
               float a[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
               if constexpr (RECON == RECON_PPM) {
                  const float fr = h4_face_fused(vm1, v0, vp1, w[q + 6]);
                  const bool fr_out = (v0 - fr) * (fr - vp1) < 0.0f;
                  const float dn = vp1 - v0;
                  const bool same = dn * dprev > 0.0f;
                  // superbee: max(min(|a|, 2|b|), min(2|a|, |b|)) = min(2 min(|a|,|b|), max(|a|,|b|))
                  const float an = fabsf(dn), ap = fabsf(dprev);
                  const float sl = fminf(2.0f * fminf(an, ap), fmaxf(an, ap));
                  const float hs = copysignf(0.5f * sl, dn);
                  float fl2 = face_out ? v0 - hs : face;
                  float fr2 = fr_out ? v0 + hs : fr;
                  fl2 = same ? fl2 : v0;
                  fr2 = same ? fr2 : v0;
                  const float d = fr2 - fl2;
                  const float ev = fmaf(-0.5f, fl2 + fr2, v0);
                  const float de = d * ev, dd = d * (d * one_sixth);
                  const float v3 = 3.0f * v0;
                  const float nfl = (de > dd) ? fmaf(-2.0f, fr2, v3) : fl2;
                  const float nfr = (-dd > de) ? fmaf(-2.0f, fl2, v3) : fr2;
                  a[0] = nfl;
                  a[1] = fmaf(-2.0f, nfl, v3) - nfr;
                  a[2] = fmaf(-2.0f, v0, nfl + nfr);
                  face = fr;
                  face_out = fr_out;
                  dprev = dn;
               } else if constexpr (RECON == RECON_PQM) {
                  const float fr = h8_value(w[q + 1], w[q + 2], w[q + 3], w[q + 4], w[q + 5], w[q + 6], w[q + 7],
                                            w[q + 8]);
                  const float fdr = h7_derivative(w[q + 1], w[q + 2], w[q + 3], w[q + 4], w[q + 5], w[q + 6],
                                                  w[q + 7], w[q + 8]);
                  pqm_coeff_fused(vm1, v0, vp1, face, fr, face_d, fdr, a);
                  face = fr;
                  face_d = fdr;
               } else {
                  plm_coeff_fused(vm1, v0, vp1, a);
               }
               // ---- distribute the cell over the lane's targets ----
               const bool has = u < 1.0f;  // the pending target's right edge lies inside this cell
               float D = recon_integral<RECON>(u, a);  // used only when has
               if (has) ring[soff] = D - nacc;
               nacc = (has ? D : nacc) - v0;
               {
                  const float g1n = g1f + 1.0f;
                  const float un = fs(fa(fm(g1n, dk), im), v_l) * inv_dv;  // the next edge (reference's rounding)
                  g1f = has ? g1n : g1f;
                  u = has ? un : u;
                  soff = has ? ((soff + 1u) & SMASK) : soff;
               }
               if (u < 1.0f) {
                  // further edges inside the same source cell (dk < dv)
                  for (int guard = 0; u < 1.0f && guard < 8; ++guard) {
                     const float D2 = recon_integral<RECON>(u, a);
                     ring[soff] = D2 - D;
                     D = D2;
                     g1f += 1.0f;
                     soff = (soff + 1u) & SMASK;
                     u = fs(fa(fm(g1f, dk), im), v_l) * inv_dv;
                  }
                  // more than eight target edges in one source cell (dk < dv / 8):
                  // outside what the walk represents, reported with the cell
                  range_err |= u < 1.0f;
                  nacc = D - v0;
               }
               u -= 1.0f;
               v_l = fa(v_l, dv);
            }
            g = __float2int_rn(g1f) - 1;  // the pending target
            int top = g - 1;  // the highest target this block completed
            if (kb == col_e) {
               // column done: the pending target keeps the rest; targets
               // above the column's highest cell are folded into it
               if (g > hi) {
                  float extra = -nacc;
                  for (int t = hi + 1; t < g && t <= hi + RING_CELLS / 2; ++t) {
                     extra += ring[t & RMASK];
                     ring[t & RMASK] = 0.0f;
                  }
                  range_err |= g > hi + RING_CELLS / 2;
                  ring[hi & RMASK] += extra;
                  top = hi;
               } else {
                  // the slot holds nothing of this column's yet (its first
                  // target's earlier content is already in nacc)
                  ring[soff] = -nacc;
                  top = g;
               }
            }
            // everything this block wrote must lie inside the ring's window
            range_err |= top >= (next_flush + RING_BLOCKS) * WID;
            // targets below the next source cell's lower bound are complete
            int lb = ncf * WID;
            if (kb < col_e) {
               int nl = __reduce_min_sync(hmask, g < hi ? g : hi);
               lb = (nl < lb) ? nl : lb;
            }
            flush_until(lb >> 2);
            pw0 = cur[0]; pw1 = cur[1]; pw2 = cur[2]; pw3 = cur[3];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
               cur[q] = nxt[q];
               nxt[q] = nn[q];
            }
            ++src_rank;
         }
         col_s = nxt_s;
         col_e = nxt_e;
         cf = ncf;
         cl = ncl;
      }
      flush_until(1 << 20);
      if (__any_sync(hmask, range_err)) {
         if (lane == 0) atomicOr(&status[cs.cell], VLGPU_CELL_RANGE);
#pragma unroll
         for (int q = 0; q < RING_CELLS; ++q) ring[q] = 0.0f;
      }
   }
}

// ---------------------------------------------------------------------------
// host-side launch helpers (used by capi.cu)
// ---------------------------------------------------------------------------
cudaError_t launch_columnize(int dim, const uint32_t* gids, const uint32_t* src_index, const CellSlot* src_slots,
                             CellSlot* dst_slots,
                             uint32_t* perm, ColumnSet* sets, uint32_t set_capacity, uint32_t dst_capacity,
                             const SweepCell* sweep_cells, uint32_t* status, SweepCounters* counters,
                             BatchStats* stats, const MeshDev& mesh, int wall_margin, uint32_t cell_begin,
                             uint32_t cell_end, int first_of_step, cudaStream_t stream) {
   uint32_t li, lj;
   plane_lengths(mesh.len, dim, li, lj);
   const size_t smem = columnize_smem_bytes(li * lj);
   const uint32_t n = cell_end - cell_begin;
   if (n == 0) return cudaSuccess;
   cudaError_t e = cudaSuccess;
#define VLGPU_COL(D)                                                                                             \
   e = cudaFuncSetAttribute(columnize_kernel<D>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);      \
   if (e != cudaSuccess) return e;                                                                              \
   columnize_kernel<D><<<n, COL_THREADS, smem, stream>>>(gids, src_index, src_slots, dst_slots, perm, sets,      \
                                                         set_capacity,                                          \
                                                         dst_capacity, sweep_cells, status, counters, stats, mesh, \
                                                         wall_margin, cell_begin, cell_end, first_of_step, nullptr, \
                                                         0xffffffffu, nullptr);
   if (dim == 0) { VLGPU_COL(0) } else if (dim == 1) { VLGPU_COL(1) } else { VLGPU_COL(2) }
#undef VLGPU_COL
   return cudaGetLastError();
}

// Columnize of every cell of a batch: one CTA per cell, the largest cells
// first (order), with shared memory for planes of up to COL_CAP_PLANE entries,
// which lets four CTAs share an SM; the cells with wider planes follow in
// columnize_wide_kernel.  The counters' n_wide must be zero (the caller clears
// the sweep counters before every sweep).
constexpr uint32_t COL_CAP_PLANE = 1024;
cudaError_t launch_columnize_batch(int dim, const uint32_t* gids, const uint32_t* src_index,
                                   const CellSlot* src_slots, CellSlot* dst_slots, uint32_t* perm, ColumnSet* sets,
                                   uint32_t set_capacity, uint32_t dst_capacity, const SweepCell* sweep_cells,
                                   uint32_t* status, SweepCounters* counters, BatchStats* stats, const MeshDev& mesh,
                                   int wall_margin, uint32_t n_cells, int first_of_step, uint32_t* wide_cells,
                                   const uint32_t* order, int wide_grid, cudaStream_t stream) {
   if (n_cells == 0) return cudaSuccess;
   uint32_t li, lj;
   plane_lengths(mesh.len, dim, li, lj);
   const uint32_t cap = li * lj < COL_CAP_PLANE ? li * lj : COL_CAP_PLANE;
   const size_t smem_cap = columnize_smem_bytes(cap);
   const size_t smem = columnize_smem_bytes(li * lj);
   const uint32_t g2 = (uint32_t)wide_grid < n_cells ? (uint32_t)wide_grid : n_cells;
   cudaError_t e = cudaSuccess;
#define VLGPU_COLB(D)                                                                                           \
   e = cudaFuncSetAttribute(columnize_kernel<D>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);       \
   if (e != cudaSuccess) return e;                                                                               \
   e = cudaFuncSetAttribute(columnize_wide_kernel<D>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);  \
   if (e != cudaSuccess) return e;                                                                               \
   columnize_kernel<D><<<n_cells, COL_THREADS, smem_cap, stream>>>(                                              \
      gids, src_index, src_slots, dst_slots, perm, sets, set_capacity, dst_capacity, sweep_cells, status, counters, \
      stats, mesh, wall_margin, 0, n_cells, first_of_step, order, cap, wide_cells);                              \
   columnize_wide_kernel<D><<<g2, COL_THREADS, smem, stream>>>(gids, src_index, src_slots, dst_slots, perm, sets, \
                                                               set_capacity, dst_capacity, sweep_cells, status,   \
                                                               counters, stats, mesh, wall_margin, first_of_step, \
                                                               wide_cells);
   if (dim == 0) { VLGPU_COLB(0) } else if (dim == 1) { VLGPU_COLB(1) } else { VLGPU_COLB(2) }
#undef VLGPU_COLB
   return cudaGetLastError();
}

// CTAs per SM of columnize_wide_kernel (the largest plane of the three
// dimensions).
int columnize_wide_blocks_per_sm(const MeshDev& mesh) {
   uint32_t li, lj, best = 0;
   for (int d = 0; d < 3; ++d) {
      plane_lengths(mesh.len, d, li, lj);
      best = li * lj > best ? li * lj : best;
   }
   const size_t smem = columnize_smem_bytes(best);
   int n = 0;
   cudaFuncSetAttribute(columnize_wide_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
   cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, columnize_wide_kernel<0>, COL_THREADS, smem);
   return n > 0 ? n : 1;
}

cudaError_t launch_remap(int dim, const ColumnSet* sets, SweepCounters* counters, const uint32_t* perm,
                         const float* src_data, float* dst_data, uint32_t* dst_gids, const SweepCell* sweep_cells,
                         uint32_t* status, const MeshDev& mesh, int wall_margin, uint32_t set_capacity,
                         uint8_t* content_out, double content_threshold, bool exact, int recon, int grid,
                         cudaStream_t stream) {
#define VLGPU_REMAP(D)                                                                                        \
   remap_kernel<D><<<grid, REMAP_THREADS, 0, stream>>>(sets, counters, perm, src_data, dst_data, dst_gids,          \
                                                       sweep_cells, status, mesh, wall_margin, set_capacity,        \
                                                       content_out, content_threshold)
#define VLGPU_WALK(D, R)                                                                                       \
   remap_walk_kernel<D, R><<<grid, REMAP_THREADS, 0, stream>>>(sets, counters, perm, src_data, dst_data, dst_gids, \
                                                               sweep_cells, status, mesh, wall_margin, set_capacity, \
                                                               content_out, content_threshold)
#define VLGPU_WALK_DIMS(R)               \
   if (dim == 0) VLGPU_WALK(0, R);       \
   else if (dim == 1) VLGPU_WALK(1, R);  \
   else VLGPU_WALK(2, R);
   if (exact) {
      if (recon != RECON_PPM) return cudaErrorInvalidValue;  // the exact mode is PPM only
      if (dim == 0) VLGPU_REMAP(0);
      else if (dim == 1) VLGPU_REMAP(1);
      else VLGPU_REMAP(2);
   } else if (recon == RECON_PLM) {
      VLGPU_WALK_DIMS(RECON_PLM)
   } else if (recon == RECON_PQM) {
      VLGPU_WALK_DIMS(RECON_PQM)
   } else {
      VLGPU_WALK_DIMS(RECON_PPM)
   }
#undef VLGPU_WALK_DIMS
#undef VLGPU_WALK
#undef VLGPU_REMAP
   return cudaGetLastError();
}

// Points the remap work counter at the first set the next columnize launch
// will create (per-cell launch sequences share one set array).
__global__ void rebase_work_kernel(SweepCounters* counters) { counters->work = counters->n_sets; }

cudaError_t launch_rebase_work(SweepCounters* counters, cudaStream_t stream) {
   rebase_work_kernel<<<1, 1, 0, stream>>>(counters);
   return cudaGetLastError();
}

int remap_blocks_per_sm() {
   int n = 0;
   cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, remap_walk_kernel<2, RECON_PPM>, REMAP_THREADS, 0);
   return n > 0 ? n : 1;
}

}  // namespace vlgpu
