// Spatial translation on a uniform periodic grid for sm_100a: one dimension of
// trans_map_1d_amr (vlasovsolver/cpu_trans_map_amr.cpp:214-443) with
// propagatePencil (:37-150), the nonuniform PPM of
// cpu_1d_ppm_nonuniform.hpp:40-62 and its h4 faces (cpu_face_estimates.hpp:
// 179-202, 327-378), and the plane skip of check_skip_remapping (:18-25).
//
// A pencil is the line of cells along the sweep dimension through one
// (transverse) cell position; all cells have width dz and target ratio 1, and
// the line wraps around periodically.  Per sweep, the union kernel and one of
// the two remap kernels run:
//
//   pencil_union_kernel   one CTA per pencil.  The union of the pencil cells'
//                         block IDs as a bitmap in shared memory; one "item"
//                         per union block ID (its ID and pencil) and, per
//                         item, the list position of that block in each cell
//                         of the pencil and its data index in the source pool
//                         (or none).
//
//   trans_fused_kernel    (fused mode, the default) one warp per item walks
//                         the whole periodic pencil in batches of 8 cells.
//                         Each lane owns two of the 64 velocity columns of the
//                         block (float2 loads: a warp reads a whole block row)
//                         and keeps a window of 14 cells in registers; each
//                         face, PPM and outgoing integral is computed once per
//                         cell (the lane's two columns packed per f32x2
//                         operation), the
//                         plane skip comes from warp ballots, and each
//                         existing block gets (own value - outgoing) + incoming
//                         from the upwind neighbour, written straight to the
//                         output pool.  The item's index tables are copied
//                         into the warp's shared-memory slice with cp.async
//                         one item ahead; no block-wide barriers.
//
//   trans_remap_kernel    (exact mode) persistent CTAs, one item at a time:
//                         the item's N blocks (zeros where a cell lacks the
//                         block) are staged in shared memory; left faces, PPM
//                         coefficients and the outgoing integral of every cell
//                         follow in passes separated by barriers.
//
// Every block of every cell belongs to exactly one item, so the output pool is
// written once per block, without atomics.
//
// In the exact mode the arithmetic follows the reference's scalar build
// operation by operation (round-to-nearest intrinsics, the same
// double-precision steps), so the result is bit-identical to the reference's
// trans_map_1d_amr.  The fused mode uses the uniform-width h4 face the
// nonuniform one reduces to, the single-precision PPM of the acceleration's
// fused mode, FMA for the outgoing integral, and no h/h ratio for equal cell
// widths.
#include <cstdint>

#include "fused_ppm.cuh"
#include "vlgpu_common.cuh"

namespace vlgpu {

constexpr uint32_t NO_ROW = 0xffffffffu;
constexpr uint32_t NO_DATA = 0xffffffffu;    // an added (all-zero) block of an adjusted list
constexpr uint32_t BAD_ITEM = 0xffffffffu;   // item slot of a pencil that did not fit
constexpr int UNION_THREADS = 512;
constexpr int TR_THREADS = 256;
constexpr uint32_t TR_MAX_N = 128;           // cells per pencil

// Counters of one translation sweep, zeroed before the union kernel.
struct TransCounters {
   uint32_t n_items;
   uint32_t work;
   uint32_t overflow;
   uint32_t pad;
};

// Constants of the nonuniform h4 face (cpu_face_estimates.hpp:179-191) for
// cells of equal width h, evaluated on the host in the reference's types.
struct FaceConsts {
   double D1, D2, D3, D4;
   float F1, F2, F3, h;
};

__device__ __forceinline__ float ta(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float ts(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float tm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float td(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float tdf(double a, double b) { return __double2float_rn(__dmul_rn(a, b)); }

// Left face of the cell whose stencil values are um2, um1, u0, up1.
__device__ __forceinline__ float face_nonuniform(const FaceConsts& c, float um2, float um1, float u0, float up1) {
   const float V1 = tm(c.F1, ta(tm(um1, c.h), tm(u0, c.h)));
   const float V2 = tdf((double)V1, c.D2);
   const float V3 = tm(c.F2, ts(tdf((double)um1, c.D3), tm(um2, c.h)));
   const float V4 = tm(c.F3, ts(tdf((double)u0, c.D4), tm(up1, c.h)));
   const float S = ta(ta(V2, V3), V4);
   return tdf(c.D1, (double)S);
}

__device__ __forceinline__ float t_minmod(float s1, float s2) {
   const float slope = (fabsf(s1) < fabsf(s2)) ? s1 : s2;
   return (tm(s1, s2) <= 0.0f) ? 0.0f : slope;
}
__device__ __forceinline__ float t_maxmod(float s1, float s2) {
   const float slope = (fabsf(s1) > fabsf(s2)) ? s1 : s2;
   return (tm(s1, s2) <= 0.0f) ? 0.0f : slope;
}

// compute_ppm_coeff_nonuniform with the filtered faces fl, fr
// (cpu_1d_ppm_nonuniform.hpp:40-62, cpu_face_estimates.hpp:327-378).
__device__ __forceinline__ void t_ppm_coeff(float vm1, float v0, float vp1, float fl, float fr, float threshold,
                                            float scale, float& a0, float& a1, float& a2) {
   const float l = tm(vm1, scale), m = tm(v0, scale), r = tm(vp1, scale);
   const float a = ts(r, m), b = ts(m, l);
   const float slope = t_maxmod(t_minmod(a, tm(2.0f, b)), t_minmod(tm(2.0f, a), b));
   const float slope_abs = tm(fabsf(slope), threshold);
   const float slope_sign = (slope > 0.0f) ? 1.0f : -1.0f;
   if (slope_abs == 0.0f) {
      fr = v0;
      fl = v0;
   }
   const float half_slope = tm(tm(slope_sign, 0.5f), slope_abs);
   if (tm(ts(vm1, fl), ts(fl, v0)) < 0.0f) fl = ts(v0, half_slope);
   if (tm(ts(vp1, fr), ts(fr, v0)) < 0.0f) fr = ta(v0, half_slope);
   const float one_sixth = (float)(1.0 / 6.0);
   {
      const float d = ts(fr, fl);
      const float e = ts(v0, tm(0.5f, ta(fl, fr)));
      if (tm(d, e) > tm(tm(d, d), one_sixth)) fl = ts(tm(3.0f, v0), tm(2.0f, fr));
   }
   {
      const float d = ts(fr, fl);
      const float e = ts(v0, tm(0.5f, ta(fl, fr)));
      if (tm(tm(-d, d), one_sixth) > tm(d, e)) fr = ts(tm(3.0f, v0), tm(2.0f, fl));
   }
   a0 = fl;
   a1 = ts(ts(tm(3.0f, v0), tm(2.0f, fl)), fr);
   a2 = ts(ta(fl, fr), tm(2.0f, v0));
}

// Cell of pencil p at position x along dimension dim (cells x fastest).
__device__ __forceinline__ uint32_t pencil_cell(uint32_t p, uint32_t x, int dim, uint32_t nx, uint32_t ny) {
   if (dim == 0) return x + nx * p;
   if (dim == 1) return (p % nx) + nx * x + nx * ny * (p / nx);
   return p + nx * ny * x;
}

// Index k (0..3) along the sweep dimension of memory offset c in a block.
template <int DIM>
__device__ __forceinline__ int plane_of(int c) {
   if (DIM == 0) return c & 3;
   if (DIM == 1) return (c >> 2) & 3;
   return c >> 4;
}

__device__ __forceinline__ uint32_t tr_exclusive_scan(uint32_t v, uint32_t* warp_sums, uint32_t& total) {
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

// ---------------------------------------------------------------------------
// pencil union: one CTA per pencil
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(UNION_THREADS) pencil_union_kernel(
   const uint32_t* __restrict__ gids, const CellSlot* __restrict__ slots, int dim, uint32_t nx, uint32_t ny,
   uint32_t N, uint32_t n_words, uint32_t* __restrict__ item_gid, uint32_t* __restrict__ item_pencil,
   uint32_t* __restrict__ rows, uint32_t* __restrict__ srcs, const uint32_t* __restrict__ src_index,
   uint32_t item_cap, uint64_t row_cap, TransCounters* __restrict__ tc, uint32_t* __restrict__ status) {
   extern __shared__ uint32_t usm[];
   uint32_t* bm = usm;             // n_words: union bitmap
   uint32_t* pre = usm + n_words;  // n_words: union entries before each word
   __shared__ uint32_t warp_sums[32];
   __shared__ uint32_t s_base;
   __shared__ int s_ok;
   const uint32_t p = blockIdx.x;
   for (uint32_t w = threadIdx.x; w < n_words; w += blockDim.x) bm[w] = 0u;
   __syncthreads();
   for (uint32_t x = 0; x < N; ++x) {
      const CellSlot s = slots[pencil_cell(p, x, dim, nx, ny)];
      for (uint32_t b = threadIdx.x; b < s.count; b += blockDim.x) {
         const uint32_t g = gids[s.off + b];
         atomicOr(&bm[g >> 5], 1u << (g & 31));
      }
   }
   __syncthreads();
   const uint32_t chunk = (n_words + blockDim.x - 1) / blockDim.x;
   const uint32_t w0 = min(n_words, threadIdx.x * chunk), w1 = min(n_words, w0 + chunk);
   uint32_t mine = 0;
   for (uint32_t w = w0; w < w1; ++w) mine += __popc(bm[w]);
   uint32_t total;
   uint32_t run = tr_exclusive_scan(mine, warp_sums, total);
   for (uint32_t w = w0; w < w1; ++w) {
      pre[w] = run;
      run += __popc(bm[w]);
   }
   if (threadIdx.x == 0) {
      const uint32_t base = atomicAdd(&tc->n_items, total);
      const bool ok = (uint64_t)base + total <= item_cap && ((uint64_t)base + total) * N <= row_cap;
      if (!ok) atomicOr(&tc->overflow, 1u);
      s_base = base;
      s_ok = ok ? 1 : 0;
   }
   __syncthreads();
   const uint32_t base = s_base;
   if (!s_ok) {
      // the reserved item slots that exist are marked unusable; the pencil's
      // cells report the shortage
      for (uint32_t r = threadIdx.x; r < total; r += blockDim.x)
         if ((uint64_t)base + r < item_cap) item_pencil[base + r] = BAD_ITEM;
      for (uint32_t x = threadIdx.x; x < N; x += blockDim.x)
         atomicOr(&status[pencil_cell(p, x, dim, nx, ny)], VLGPU_CELL_NOMEM);
      return;
   }
   for (uint32_t w = w0; w < w1; ++w) {
      uint32_t m = bm[w];
      uint32_t r = pre[w];
      while (m) {
         const int bit = __ffs(m) - 1;
         m &= m - 1;
         item_gid[base + r] = w * 32u + (uint32_t)bit;
         item_pencil[base + r] = p;
         ++r;
      }
   }
   const uint64_t row0 = (uint64_t)base * N;
   for (uint64_t e = threadIdx.x; e < (uint64_t)total * N; e += blockDim.x) {
      rows[row0 + e] = NO_ROW;
      srcs[row0 + e] = NO_DATA;
   }
   __syncthreads();
   for (uint32_t x = 0; x < N; ++x) {
      const CellSlot s = slots[pencil_cell(p, x, dim, nx, ny)];
      for (uint32_t b = threadIdx.x; b < s.count; b += blockDim.x) {
         const uint32_t g = gids[s.off + b];
         const uint32_t w = g >> 5;
         const uint32_t r = pre[w] + __popc(bm[w] & ((1u << (g & 31)) - 1u));
         rows[row0 + (uint64_t)r * N + x] = s.off + b;
         srcs[row0 + (uint64_t)r * N + x] = src_index ? src_index[s.off + b] : s.off + b;
      }
   }
}

// ---------------------------------------------------------------------------
// exact translation remap: persistent CTAs, one item (pencil, block ID) at a time
// ---------------------------------------------------------------------------
template <int DIM>
__global__ void __launch_bounds__(TR_THREADS) trans_remap_kernel(
   const uint32_t* __restrict__ item_gid, const uint32_t* __restrict__ item_pencil, const uint32_t* __restrict__ rows,
   TransCounters* __restrict__ tc, uint32_t item_cap, const uint32_t* __restrict__ src_index,
   const float* __restrict__ src, float* __restrict__ dst, uint32_t* __restrict__ dst_gids, MeshDev mesh,
   uint32_t N, FaceConsts fc, float dt, float threshold, float scale) {
   extern __shared__ float tsm[];
   const uint32_t NE = N * WID3;
   float* V = tsm;                          // values of the item's blocks, [x][c]
   float* NB = tsm + NE;                    // outgoing integral (ngbr) of every cell
   float* F = tsm + 2 * NE;                 // left face of every cell
   __shared__ uint32_t s_row[TR_MAX_N];
   __shared__ uint32_t s_pos[TR_MAX_N];  // bit k: some value of plane k of block x is positive
   __shared__ uint32_t s_item;
   __shared__ float s_z1[WID], s_z2[WID];
   __shared__ int s_up[WID];
   const int lane = threadIdx.x & 31;
   uint32_t n_items = *((volatile uint32_t*)&tc->n_items);
   n_items = (n_items < item_cap) ? n_items : item_cap;
   const float dvz = mesh.dv[DIM], vz_min = mesh.vmin[DIM];

   for (;;) {
      if (threadIdx.x == 0) s_item = atomicAdd(&tc->work, 1u);
      __syncthreads();
      const uint32_t q = s_item;
      if (q >= n_items) break;
      const uint32_t pencil = item_pencil[q];
      if (pencil == BAD_ITEM) {
         __syncthreads();
         continue;
      }
      const uint32_t gid = item_gid[q];
      for (uint32_t x = threadIdx.x; x < N; x += blockDim.x) {
         s_row[x] = rows[(uint64_t)q * N + x];
         s_pos[x] = 0u;
      }
      if (threadIdx.x < WID) {
         // Lagrangian shift of plane k (cpu_trans_map_amr.cpp:60-80)
         uint32_t sw[3];
         swapped_indices(gid, mesh.len, DIM, sw);
         const int k = threadIdx.x;
         const float cell_vz = __double2float_rn(((double)(sw[2] * WID + k) + 0.5) * (double)dvz + (double)vz_min);
         const float zt = td(tm(cell_vz, dt), fc.h);
         const bool up = zt > 0.0f;
         s_z1[k] = up ? __double2float_rn(1.0 - (double)zt) : 0.0f;
         s_z2[k] = up ? 1.0f : -zt;
         s_up[k] = up ? 1 : 0;
      }
      __syncthreads();
      // pass 1: stage the values; positive-value flags per (block, plane)
      for (uint32_t e = threadIdx.x; e < NE; e += blockDim.x) {
         const uint32_t x = e >> 6;
         const int c = (int)(e & 63);
         const uint32_t r = s_row[x];
         float v = 0.0f;
         if (r != NO_ROW) {
            const uint32_t idx = src_index ? src_index[r] : r;
            if (idx != NO_DATA) v = src[(size_t)idx * WID3 + c];
         }
         V[e] = v;
         const int k = plane_of<DIM>(c);
         uint32_t bits = 0;
#pragma unroll
         for (int kk = 0; kk < WID; ++kk)
            if (__any_sync(0xffffffffu, (v > 0.0f) && (k == kk))) bits |= 1u << kk;
         if (lane == 0 && bits) atomicOr(&s_pos[x], bits);
      }
      __syncthreads();
      // pass 2: left faces
      for (uint32_t e = threadIdx.x; e < NE; e += blockDim.x) {
         const uint32_t x = e >> 6, c = e & 63;
         const uint32_t xm2 = (x + 2 * N - 2) % N, xm1 = (x + N - 1) % N, xp1 = (x + 1) % N;
         F[e] = face_nonuniform(fc, V[xm2 * WID3 + c], V[xm1 * WID3 + c], V[e], V[xp1 * WID3 + c]);
      }
      __syncthreads();
      // pass 3: PPM coefficients and the integral leaving each cell, for the
      // planes that are not skipped
      for (uint32_t e = threadIdx.x; e < NE; e += blockDim.x) {
         const uint32_t x = e >> 6, c = e & 63;
         const int k = plane_of<DIM>((int)c);
         const uint32_t xm2 = (x + 2 * N - 2) % N, xm1 = (x + N - 1) % N, xp1 = (x + 1) % N, xp2 = (x + 2) % N;
         const uint32_t act = (s_pos[xm2] | s_pos[xm1] | s_pos[x] | s_pos[xp1] | s_pos[xp2]) >> k & 1u;
         float ngbr = 0.0f;
         if (act) {
            float a0, a1, a2;
            const float z1 = s_z1[k], z2 = s_z2[k];
            t_ppm_coeff(V[xm1 * WID3 + c], V[e], V[xp1 * WID3 + c], F[e], F[xp1 * WID3 + c], threshold, scale, a0,
                        a1, a2);
            const float i2 = tm(z2, ta(a0, tm(z2, ta(a1, tm(z2, a2)))));
            const float i1 = tm(z1, ta(a0, tm(z1, ta(a1, tm(z1, a2)))));
            ngbr = ts(i2, i1);
         }
         NB[e] = ngbr;
      }
      __syncthreads();
      // pass 4: the new values of the blocks that exist
      for (uint32_t e = threadIdx.x; e < NE; e += blockDim.x) {
         const uint32_t x = e >> 6, c = e & 63;
         const uint32_t r = s_row[x];
         if (r == NO_ROW) continue;
         const int k = plane_of<DIM>((int)c);
         const uint32_t xm1 = (x + N - 1) % N, xp1 = (x + 1) % N;
         const uint32_t xm2 = (x + 2 * N - 2) % N, xp2 = (x + 2) % N;
         const uint32_t xm3 = (x + 3 * N - 3) % N, xp3 = (x + 3) % N;
         const uint32_t act_self = (s_pos[xm2] | s_pos[xm1] | s_pos[x] | s_pos[xp1] | s_pos[xp2]) >> k & 1u;
         float out = 0.0f;
         if (act_self) out = ta(out, ts(V[e], NB[e]));
         if (s_up[k]) {
            const uint32_t act = (s_pos[xm3] | s_pos[xm2] | s_pos[xm1] | s_pos[x] | s_pos[xp1]) >> k & 1u;
            if (act) out = ta(out, td(tm(NB[xm1 * WID3 + c], fc.h), fc.h));
         } else {
            const uint32_t act = (s_pos[xm1] | s_pos[x] | s_pos[xp1] | s_pos[xp2] | s_pos[xp3]) >> k & 1u;
            if (act) out = ta(out, td(tm(NB[xp1 * WID3 + c], fc.h), fc.h));
         }
         dst[(size_t)r * WID3 + c] = out;
         if (c == 0) dst_gids[r] = gid;
      }
      __syncthreads();
   }
}

// ---------------------------------------------------------------------------
// fused translation remap: one warp per item (pencil, block ID)
// ---------------------------------------------------------------------------
constexpr int TF_THREADS = 256;
constexpr int TF_BATCH = 8;  // cells per batch of the walk (16 measured slower)

// Lanes whose columns share the plane (index along the sweep dimension) of
// this lane's first column; a lane owns columns 2 lane and 2 lane + 1.  For
// DIM 0 the second column lies in the next plane, with the same lanes.
template <int DIM>
__device__ __forceinline__ uint32_t plane_lanes(int lane) {
   if (DIM == 0) return (lane & 1) ? 0xaaaaaaaau : 0x55555555u;
   if (DIM == 1) return 0x03030303u << (2 * ((lane >> 1) & 3));
   return 0xffu << (8 * (lane >> 3));
}
template <int DIM>
__device__ __forceinline__ int lane_plane(int lane) {
   if (DIM == 0) return 2 * (lane & 1);
   if (DIM == 1) return (lane >> 1) & 3;
   return lane >> 3;
}

// Shift of plane k of the block at swapped index sw2 along the sweep
// dimension, as fractions of the cell: outgoing integral over [z1, z2]
// (cpu_trans_map_amr.cpp:60-80; fused arithmetic).
__device__ __forceinline__ void plane_shift(uint32_t sw2, int k, float dvz, float vz_min, float dt, float h,
                                            float& z1, float& z2, bool& up) {
   const float cell_vz = __double2float_rn(((double)(sw2 * WID + k) + 0.5) * (double)dvz + (double)vz_min);
   const float zt = __fdiv_rn(__fmul_rn(cell_vz, dt), h);
   up = zt > 0.0f;
   z1 = up ? 1.0f - zt : 0.0f;
   z2 = up ? 1.0f : -zt;
}

// The PPM (ppm_coeff_x2) and the outgoing integral over [z1, z2] of two
// columns given their left and right faces; zero for a column whose plane is
// skipped.
__device__ __forceinline__ float2 outgoing_x2(float2 vm1, float2 v0, float2 vp1, float2 fl, float2 fr, float2 z1,
                                              float2 z2, uint32_t act_x, uint32_t act_y) {
   float2 a0, a1, a2;
   ppm_coeff_x2(vm1, v0, vp1, fl, fr, a0, a1, a2);
   const float2 t2 = __ffma2_rn(z2, __ffma2_rn(z2, a2, a1), a0);
   const float2 t1 = __ffma2_rn(z1, __ffma2_rn(z1, a2, a1), a0);
   const float2 ngbr = p_sub(__fmul2_rn(z2, t2), __fmul2_rn(z1, t1));
   return make_float2(act_x ? ngbr.x : 0.0f, act_y ? ngbr.y : 0.0f);
}

// The same in the walk form (ppm_walk_x2): the left-face test and v0 - vm1
// come in from the cell to the left, and this cell's go out in tl and dprev.
__device__ __forceinline__ float2 outgoing_walk_x2(float2 v0, float2 vp1, float2 fl, float2 fr, float2& tl,
                                                   float2& dprev, float2 z1, float2 z2, uint32_t act_x,
                                                   uint32_t act_y) {
   float2 a0, a1, a2, tr, dn;
   ppm_walk_x2(v0, vp1, fl, fr, tl, dprev, tr, dn, a0, a1, a2);
   tl = tr;
   dprev = dn;
   const float2 t2 = __ffma2_rn(z2, __ffma2_rn(z2, a2, a1), a0);
   const float2 t1 = __ffma2_rn(z1, __ffma2_rn(z1, a2, a1), a0);
   const float2 ngbr = p_sub(__fmul2_rn(z2, t2), __fmul2_rn(z1, t1));
   return make_float2(act_x ? ngbr.x : 0.0f, act_y ? ngbr.y : 0.0f);
}

// This lane's two columns of the block at data index idx (zeros where the
// cell lacks the block).
__device__ __forceinline__ float2 load_column_pair(const float* __restrict__ src, uint32_t idx, int lane) {
   return (idx != NO_DATA) ? reinterpret_cast<const float2*>(src + (size_t)idx * WID3)[lane]
                           : make_float2(0.0f, 0.0f);
}

// px (py) = 1 when the plane of this lane's first (second) column holds a
// positive value in this cell's block, over the whole warp.
template <int DIM>
__device__ __forceinline__ void plane_positive(float2 v, uint32_t pmask, uint32_t& px, uint32_t& py) {
   if (DIM == 0) {
      px = (__ballot_sync(0xffffffffu, v.x > 0.0f) & pmask) != 0u;
      py = (__ballot_sync(0xffffffffu, v.y > 0.0f) & pmask) != 0u;
   } else {
      px = (__ballot_sync(0xffffffffu, (v.x > 0.0f) | (v.y > 0.0f)) & pmask) != 0u;
      py = px;
   }
}

// One warp per item walks the whole (periodic) pencil, L cells per batch.
// Window index of cell c in the batch that outputs cells s0 .. s0+L-1 is
// c - s0 + 3; the window holds cells s0-3 .. s0+L+2, the first six carried
// over from the previous batch.  Carried along the walk: the left face fl of
// the next cell and the outgoing integrals nb_m1, nb_0 of the two cells before
// it, so every face and PPM is evaluated once per cell (plus two at the start).
//
// The item's header and tables live in the warp's slice of shared memory,
// double-buffered: [0] pencil, [1] block ID, tsrc[m] (m = 0 .. N+5) = data
// index of cell (m - 3) mod N (window order, no wrap at use) and trow[x] =
// list row of output cell x.  The next item's slice is copied in with
// cp.async while the current item is computed, so only the data loads wait on
// memory.
__device__ __forceinline__ void cp_async4(uint32_t* smem_dst, const uint32_t* gmem_src) {
   asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((uint32_t)__cvta_generic_to_shared(smem_dst)),
                "l"(gmem_src)
                : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
   asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

__host__ __device__ constexpr uint32_t tf_slice_words(uint32_t N) { return 2 * N + 8; }

template <int DIM, int L>
__global__ void __launch_bounds__(TF_THREADS, 3) trans_fused_kernel(
   const uint32_t* __restrict__ item_gid, const uint32_t* __restrict__ item_pencil, const uint32_t* __restrict__ rows,
   const uint32_t* __restrict__ srcs, const TransCounters* __restrict__ tc, uint32_t item_cap, uint64_t row_cap,
   const float* __restrict__ src, float* __restrict__ dst, uint32_t* __restrict__ dst_gids, MeshDev mesh,
   uint32_t N, float dt, float h) {
   constexpr int W = L + 6;
   extern __shared__ uint32_t tf_smem[];
   const int lane = threadIdx.x & 31;
   uint32_t* const slices = tf_smem + (threadIdx.x >> 5) * 2 * tf_slice_words(N);
   const uint32_t warp0 = (blockIdx.x * TF_THREADS + threadIdx.x) >> 5;
   const uint32_t n_warps = (gridDim.x * TF_THREADS) >> 5;
   uint32_t n_items = *((const volatile uint32_t*)&tc->n_items);
   n_items = (n_items < item_cap) ? n_items : item_cap;
   const uint32_t pmask = plane_lanes<DIM>(lane);
   const int kx = lane_plane<DIM>(lane), ky = (DIM == 0) ? kx + 1 : kx;
   const float dvz = mesh.dv[DIM], vz_min = mesh.vmin[DIM];

   // copy item q's header and tables into slice sl (entries past row_cap, of
   // an item whose pencil did not fit, read as none)
   auto prefetch = [&](uint32_t q, uint32_t* sl) {
      if (q >= n_items) {
         if (lane == 0) sl[0] = BAD_ITEM;
         return;
      }
      if (lane == 0) {
         cp_async4(sl, item_pencil + q);
         cp_async4(sl + 1, item_gid + q);
      }
      const uint64_t base = (uint64_t)q * N;
      for (uint32_t m = lane; m < N + 6; m += 32) {
         const uint32_t cell = (m + 3u * N - 3u) % N;
         if (base + cell < row_cap) cp_async4(sl + 2 + m, srcs + base + cell);
         else sl[2 + m] = NO_DATA;
      }
      for (uint32_t m = lane; m < N; m += 32) {
         if (base + m < row_cap) cp_async4(sl + N + 8 + m, rows + base + m);
         else sl[N + 8 + m] = NO_ROW;
      }
      cp_async_commit();
   };

   prefetch(warp0, slices);
   uint32_t parity = 0;
   for (uint32_t q = warp0; q < n_items; q += n_warps, parity ^= 1u) {
      cp_async_wait_all();
      __syncwarp();
      const uint32_t* const sl = slices + parity * tf_slice_words(N);
      const uint32_t* const tsrc = sl + 2;
      const uint32_t* const trow = sl + N + 8;
      const uint32_t pencil = sl[0], gid = sl[1];
      prefetch(q + n_warps, slices + (parity ^ 1u) * tf_slice_words(N));
      if (pencil == BAD_ITEM) continue;

      uint32_t sw[3];
      swapped_indices(gid, mesh.len, DIM, sw);
      float2 z1, z2;
      bool upx, upy;
      plane_shift(sw[2], kx, dvz, vz_min, dt, h, z1.x, z2.x, upx);
      plane_shift(sw[2], ky, dvz, vz_min, dt, h, z1.y, z2.y, upy);

      // window cells -3 .. L+2 of the first batch (past N+2: not needed)
      float2 w[W];
      uint32_t posx = 0u, posy = 0u;  // bit j: positive value in window cell j
#pragma unroll
      for (int j = 0; j < W; ++j) w[j] = load_column_pair(src, ((uint32_t)j < N + 6) ? tsrc[j] : NO_DATA, lane);
#pragma unroll
      for (int j = 0; j < W; ++j) {
         uint32_t px, py;
         plane_positive<DIM>(w[j], pmask, px, py);
         posx |= px << j;
         posy |= py << j;
      }
      // the outgoing integrals of cells -1 and 0, the left face of cell 1
      // and, carried along the walk, its left-face test and v0 - vm1
      float2 nb_m1, nb_0, fl, tl, dprev;
      {
         const uint32_t ax = posx | (posx << 1) | (posx << 2) | (posx >> 1) | (posx >> 2);
         const uint32_t ay = posy | (posy << 1) | (posy << 2) | (posy >> 1) | (posy >> 2);
         const float2 fm1 = h4_face_x2(w[0], w[1], w[2], w[3]);
         const float2 f0 = h4_face_x2(w[1], w[2], w[3], w[4]);
         fl = h4_face_x2(w[2], w[3], w[4], w[5]);
         tl = __fmul2_rn(p_sub(w[1], fm1), p_sub(fm1, w[2]));
         dprev = p_sub(w[2], w[1]);
         nb_m1 = outgoing_walk_x2(w[2], w[3], fm1, f0, tl, dprev, z1, z2, (ax >> 2) & 1u, (ay >> 2) & 1u);
         nb_0 = outgoing_walk_x2(w[3], w[4], f0, fl, tl, dprev, z1, z2, (ax >> 3) & 1u, (ay >> 3) & 1u);
      }

      for (uint32_t s0 = 0;;) {
         // bit j: some positive value in window cells j-2 .. j+2 (the plane is
         // remapped for that cell; check_skip_remapping)
         const uint32_t ax = posx | (posx << 1) | (posx << 2) | (posx >> 1) | (posx >> 2);
         const uint32_t ay = posy | (posy << 1) | (posy << 2) | (posy >> 1) | (posy >> 2);
#pragma unroll
         for (int i = 0; i < L; ++i) {
            // cell y = s0+1+i (window i+4): its right face and outgoing integral;
            // then the new value of cell y-1 = s0+i (window i+3)
            const float2 fr = h4_face_x2(w[i + 3], w[i + 4], w[i + 5], w[i + 6]);
            const float2 nb = outgoing_walk_x2(w[i + 4], w[i + 5], fl, fr, tl, dprev, z1, z2, (ax >> (i + 4)) & 1u,
                                               (ay >> (i + 4)) & 1u);
            fl = fr;
            const uint32_t r = (s0 + (uint32_t)i < N) ? trow[s0 + i] : NO_ROW;
            if (r != NO_ROW) {
               float2 out;
               out.x = ((ax >> (i + 3)) & 1u) ? w[i + 3].x - nb_0.x : 0.0f;
               out.y = ((ay >> (i + 3)) & 1u) ? w[i + 3].y - nb_0.y : 0.0f;
               out.x = out.x + (upx ? nb_m1.x : nb.x);
               out.y = out.y + (upy ? nb_m1.y : nb.y);
               reinterpret_cast<float2*>(dst + (size_t)r * WID3)[lane] = out;
               if (lane == 0) dst_gids[r] = gid;
            }
            nb_m1 = nb_0;
            nb_0 = nb;
         }
         s0 += L;
         if (s0 >= N) break;
         // next batch: carry six cells, load cells s0+3 .. s0+L+2
#pragma unroll
         for (int j = 0; j < 6; ++j) w[j] = w[L + j];
         posx >>= L;
         posy >>= L;
#pragma unroll
         for (int j = 0; j < L; ++j) {
            const uint32_t m = s0 + 6u + (uint32_t)j;
            w[6 + j] = load_column_pair(src, (m < N + 6) ? tsrc[m] : NO_DATA, lane);
         }
#pragma unroll
         for (int j = 0; j < L; ++j) {
            uint32_t px, py;
            plane_positive<DIM>(w[6 + j], pmask, px, py);
            posx |= px << (6 + j);
            posy |= py << (6 + j);
         }
      }
   }
}

// ---------------------------------------------------------------------------
// host-side launch helpers
// ---------------------------------------------------------------------------
FaceConsts face_consts(float h) {
   // the reference's nonuniform face with h[-2..1] all equal to h
   volatile float hv = h;
   const float h2 = hv + hv, h3 = h2 + hv, h4 = h3 + hv;
   FaceConsts c;
   c.h = h;
   c.D1 = 1.0 / (double)h4;
   c.F1 = (h2 * h2) / h2;
   c.D2 = 1.0 / (double)h3 + 1.0 / (double)h3;
   c.F2 = (hv * h2) / (h3 * h2);
   c.D3 = (double)hv + 2.0 * (double)hv;
   c.F3 = (hv * h2) / (h3 * h2);
   c.D4 = 2.0 * (double)hv + (double)hv;
   return c;
}

uint32_t union_words(const MeshDev& mesh) { return (mesh.len[0] * mesh.len[1] * mesh.len[2] + 31) / 32; }

cudaError_t launch_pencil_union(const uint32_t* gids, const CellSlot* slots, int dim, uint32_t nx, uint32_t ny,
                                uint32_t nz, const MeshDev& mesh, uint32_t* item_gid, uint32_t* item_pencil,
                                uint32_t* rows, uint32_t* srcs, const uint32_t* src_index, uint32_t item_cap,
                                uint64_t row_cap, TransCounters* tc, uint32_t* status, cudaStream_t stream) {
   const uint32_t dims[3] = {nx, ny, nz};
   const uint32_t N = dims[dim];
   const uint32_t n_pencils = nx * ny * nz / N;
   const uint32_t n_words = union_words(mesh);
   const size_t smem = sizeof(uint32_t) * 2 * (size_t)n_words;
   cudaError_t e = cudaFuncSetAttribute(pencil_union_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
   if (e != cudaSuccess) return e;
   pencil_union_kernel<<<n_pencils, UNION_THREADS, smem, stream>>>(gids, slots, dim, nx, ny, N, n_words, item_gid,
                                                                     item_pencil, rows, srcs, src_index, item_cap,
                                                                     row_cap, tc, status);
   return cudaGetLastError();
}

size_t trans_smem_bytes(uint32_t N, bool exact) { return exact ? sizeof(float) * 3 * (size_t)N * WID3 : 0; }

size_t trans_fused_smem_bytes(uint32_t N) { return sizeof(uint32_t) * (TF_THREADS / 32) * 2 * tf_slice_words(N); }

int trans_blocks_per_sm(uint32_t N, bool exact) {
   int n = 0;
   if (exact) {
      const size_t smem = trans_smem_bytes(N, exact);
      cudaFuncSetAttribute(trans_remap_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, trans_remap_kernel<0>, TR_THREADS, smem);
   } else {
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, trans_fused_kernel<0, TF_BATCH>, TF_THREADS,
                                                    trans_fused_smem_bytes(N));
   }
   return n > 0 ? n : 1;
}

cudaError_t launch_trans_remap(int dim, uint32_t N, const uint32_t* item_gid, const uint32_t* item_pencil,
                               const uint32_t* rows, const uint32_t* srcs, TransCounters* tc, uint32_t item_cap,
                               uint64_t row_cap, const uint32_t* src_index, const float* src, float* dst,
                               uint32_t* dst_gids, const MeshDev& mesh, float dt, float dz, float threshold, bool exact,
                               int grid, cudaStream_t stream) {
   if (!exact) {
      const size_t smem = trans_fused_smem_bytes(N);
#define VLGPU_TF(D, L)                                                                                    \
   trans_fused_kernel<D, L><<<grid, TF_THREADS, smem, stream>>>(item_gid, item_pencil, rows, srcs, tc, item_cap, \
                                                                row_cap, src, dst, dst_gids, mesh, N, dt, dz);
      if (dim == 0) { VLGPU_TF(0, TF_BATCH) } else if (dim == 1) { VLGPU_TF(1, TF_BATCH) } else { VLGPU_TF(2, TF_BATCH) }
#undef VLGPU_TF
      return cudaGetLastError();
   }
   const FaceConsts fc = face_consts(dz);
   const float scale = (float)(1.0 / (double)threshold);
   const size_t smem = trans_smem_bytes(N, exact);
   cudaError_t e = cudaSuccess;
#define VLGPU_TR(D)                                                                                              \
   e = cudaFuncSetAttribute(trans_remap_kernel<D>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);      \
   if (e != cudaSuccess) return e;                                                                               \
   trans_remap_kernel<D><<<grid, TR_THREADS, smem, stream>>>(item_gid, item_pencil, rows, tc, item_cap, src_index, \
                                                             src, dst, dst_gids, mesh, N, fc, dt, threshold, scale);
   if (dim == 0) { VLGPU_TR(0) } else if (dim == 1) { VLGPU_TR(1) } else { VLGPU_TR(2) }
#undef VLGPU_TR
   return cudaGetLastError();
}

}  // namespace vlgpu
