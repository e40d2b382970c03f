// Velocity moments (FP64, Kahan-compensated) and the per-cell FP64
// acceleration geometry, for sm_100a.
//
// moments_kernel: one CTA per cell.  Each thread owns one of the 64 cells
// of a block (so its velocity offset inside the block is fixed) and walks
// the cell's blocks with a stride; its partial sums are Kahan-compensated
// doubles, merged across the CTA with error-free (TwoSum) additions.  The
// sums are those of blockVelocityFirstMoments / blockVelocitySecondMoments
// (vlasovsolver/arch_moments.h:83-155) and the per-cell bookkeeping of
// calculateMoments_V (vlasovsolver/arch_moments.cpp:342-499).
//
// geometry_kernel: one thread per cell builds the gyration transform and the
// three intersection sets in FP64 (geometry.cuh) and converts them into the
// Realf sweep parameters of the three sweeps.
#include <cstdint>

#include "geometry.cuh"
#include "vlgpu_common.cuh"

namespace vlgpu {

// Per-cell moment record (doubles).
enum MomentSlot {
   MOM_N = 0,     // sum f dv^3        (array[0])
   MOM_NVX = 1,   // sum f vx dv^3     (array[1])
   MOM_NVY = 2,
   MOM_NVZ = 3,
   MOM_RHOM = 4,  // RHOM_V = n * mass
   MOM_VX = 5,    // VX_V
   MOM_VY = 6,
   MOM_VZ = 7,
   MOM_RHOQ = 8,  // RHOQ_V = n * charge
   MOM_P11 = 9,   // P_11_V .. P_12_V = mass * sum f (v-V)(v-V) dv^3
   MOM_P22 = 10,
   MOM_P33 = 11,
   MOM_P23 = 12,
   MOM_P13 = 13,
   MOM_P12 = 14,
   MOM_MASS = 15, // plain sum of f (for conservation checks)
   MOM_COUNT = 16
};

struct Kahan {
   double s = 0.0, c = 0.0;
   __device__ __forceinline__ void add(double x) {
      const double y = x - c;
      const double t = s + y;
      c = (t - s) - y;
      s = t;
   }
};

// error-free merge of two compensated sums (Knuth TwoSum on the heads)
__device__ __forceinline__ void dd_add(double& hi, double& lo, double bhi, double blo) {
   const double s = hi + bhi;
   const double bb = s - hi;
   const double err = (hi - (s - bb)) + (bhi - bb);
   hi = s;
   lo = lo + blo + err;
}

constexpr int MOM_THREADS = 256;

template <int N>
__device__ __forceinline__ void cta_reduce(double hi[N], double lo[N], double* sh_hi, double* sh_lo) {
   // warp level
#pragma unroll
   for (int q = 0; q < N; ++q) {
#pragma unroll
      for (int o = 16; o >= 1; o >>= 1) {
         const double oh = __shfl_xor_sync(0xffffffffu, hi[q], o);
         const double ol = __shfl_xor_sync(0xffffffffu, lo[q], o);
         dd_add(hi[q], lo[q], oh, ol);
      }
   }
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
   if (lane == 0)
      for (int q = 0; q < N; ++q) {
         sh_hi[warp * N + q] = hi[q];
         sh_lo[warp * N + q] = lo[q];
      }
   __syncthreads();
   if (threadIdx.x == 0) {
      for (int q = 0; q < N; ++q) {
         double h = 0.0, l = 0.0;
         for (int w = 0; w < MOM_THREADS / 32; ++w) dd_add(h, l, sh_hi[w * N + q], sh_lo[w * N + q]);
         hi[q] = h;
         lo[q] = l;
      }
   }
   __syncthreads();
}

__global__ void __launch_bounds__(MOM_THREADS) moments_kernel(
   const uint32_t* __restrict__ gids, const uint32_t* __restrict__ src_index, const float* __restrict__ data,
   const CellSlot* __restrict__ slots, double* __restrict__ moments, MeshDev mesh, double vmin0, double vmin1, double vmin2, double bs0, double bs1,
   double bs2, double dv0, double dv1, double dv2, double mass, double charge, int second) {
   __shared__ double sh_hi[(MOM_THREADS / 32) * 6];
   __shared__ double sh_lo[(MOM_THREADS / 32) * 6];
   __shared__ double s_V[3];
   const uint32_t cell = blockIdx.x;
   const CellSlot s = slots[cell];
   double* out = moments + (size_t)cell * MOM_COUNT;
   const int ci = threadIdx.x & 63;
   const int i = ci & 3, j = (ci >> 2) & 3, k = ci >> 4;
   const double DV3 = dv0 * dv1 * dv2;
   const double HALF = 0.5;
   Kahan acc[5];
   for (uint32_t b = threadIdx.x >> 6; b < s.count; b += MOM_THREADS / 64) {
      const uint32_t gid = gids[s.off + b];
      const uint32_t bi = gid % mesh.len[0], bj = (gid / mesh.len[0]) % mesh.len[1];
      const uint32_t bk = gid / (mesh.len[0] * mesh.len[1]);
      const double VX = (vmin0 + bi * bs0) + (i + HALF) * dv0;
      const double VY = (vmin1 + bj * bs1) + (j + HALF) * dv1;
      const double VZ = (vmin2 + bk * bs2) + (k + HALF) * dv2;
      const uint32_t idx = src_index ? src_index[s.off + b] : s.off + b;
      if (idx == 0xffffffffu) continue;  // an added block holds zeros
      const double f = (double)data[(size_t)idx * WID3 + ci];
      acc[0].add(f * DV3);
      acc[1].add(f * VX * DV3);
      acc[2].add(f * VY * DV3);
      acc[3].add(f * VZ * DV3);
      acc[4].add(f);
   }
   double hi[6], lo[6];
   for (int q = 0; q < 5; ++q) {
      hi[q] = acc[q].s;
      lo[q] = -acc[q].c;
   }
   hi[5] = lo[5] = 0.0;
   cta_reduce<5>(hi, lo, sh_hi, sh_lo);
   if (threadIdx.x == 0) {
      const double a0 = hi[0] + lo[0], a1 = hi[1] + lo[1], a2 = hi[2] + lo[2], a3 = hi[3] + lo[3];
      out[MOM_N] = a0;
      out[MOM_NVX] = a1;
      out[MOM_NVY] = a2;
      out[MOM_NVZ] = a3;
      const double rhom = a0 * mass;
      out[MOM_RHOM] = rhom;
      const double vx = (rhom != 0.0) ? (a1 * mass) / rhom : 0.0;
      const double vy = (rhom != 0.0) ? (a2 * mass) / rhom : 0.0;
      const double vz = (rhom != 0.0) ? (a3 * mass) / rhom : 0.0;
      out[MOM_VX] = vx;
      out[MOM_VY] = vy;
      out[MOM_VZ] = vz;
      out[MOM_RHOQ] = a0 * charge;
      out[MOM_MASS] = hi[4] + lo[4];
      s_V[0] = vx;
      s_V[1] = vy;
      s_V[2] = vz;
   }
   if (!second) return;
   __syncthreads();
   const double aVX = s_V[0], aVY = s_V[1], aVZ = s_V[2];
   Kahan p[6];
   for (uint32_t b = threadIdx.x >> 6; b < s.count; b += MOM_THREADS / 64) {
      const uint32_t gid = gids[s.off + b];
      const uint32_t bi = gid % mesh.len[0], bj = (gid / mesh.len[0]) % mesh.len[1];
      const uint32_t bk = gid / (mesh.len[0] * mesh.len[1]);
      const double VX = (vmin0 + bi * bs0) + (i + HALF) * dv0;
      const double VY = (vmin1 + bj * bs1) + (j + HALF) * dv1;
      const double VZ = (vmin2 + bk * bs2) + (k + HALF) * dv2;
      const uint32_t idx = src_index ? src_index[s.off + b] : s.off + b;
      if (idx == 0xffffffffu) continue;
      const double f = (double)data[(size_t)idx * WID3 + ci];
      p[0].add(f * (VX - aVX) * (VX - aVX) * DV3);
      p[1].add(f * (VY - aVY) * (VY - aVY) * DV3);
      p[2].add(f * (VZ - aVZ) * (VZ - aVZ) * DV3);
      p[3].add(f * (VY - aVY) * (VZ - aVZ) * DV3);
      p[4].add(f * (VX - aVX) * (VZ - aVZ) * DV3);
      p[5].add(f * (VX - aVX) * (VY - aVY) * DV3);
   }
   for (int q = 0; q < 6; ++q) {
      hi[q] = p[q].s;
      lo[q] = -p[q].c;
   }
   cta_reduce<6>(hi, lo, sh_hi, sh_lo);
   if (threadIdx.x == 0)
      for (int q = 0; q < 6; ++q) out[MOM_P11 + q] = mass * (hi[q] + lo[q]);
}

// Per-cell acceleration inputs on the device.
struct CellAccelInputs {
   double B[3];
   double curl[3];
   double egradpe[3];
   double dt;
};

__global__ void geometry_kernel(const CellAccelInputs* __restrict__ in, const double* __restrict__ moments,
                                double* __restrict__ isect12, SweepCell* __restrict__ sweep3, uint32_t n_cells,
                                double q, double m, double hall_min_rhoq, int ohm_gradpe, double mu0, double vmin0,
                                double vmin1, double vmin2, double dv0, double dv1, double dv2, uint32_t map_order,
                                float threshold) {
   const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
   if (c >= n_cells) return;
   const CellAccelInputs a = in[c];
   const double* mom = moments + (size_t)c * MOM_COUNT;
   geom::TransformInputs ti;
   for (int r = 0; r < 3; ++r) {
      ti.B[r] = a.B[r];
      ti.curl[r] = a.curl[r];
      ti.egradpe[r] = a.egradpe[r];
   }
   ti.V[0] = mom[MOM_VX];
   ti.V[1] = mom[MOM_VY];
   ti.V[2] = mom[MOM_VZ];
   ti.rhoq = mom[MOM_RHOQ];
   ti.q = q;
   ti.m = m;
   ti.dt = a.dt;
   ti.hall_min_rhoq = hall_min_rhoq;
   ti.ohm_gradpe = ohm_gradpe;
   ti.mu0 = mu0;
   const geom::Affine T = geom::acceleration_transform(ti);
   const double mn[3] = {vmin0, vmin1, vmin2};
   const double dv[3] = {dv0, dv1, dv2};
   double* I = isect12 + (size_t)c * 12;
   geom::cell_intersections(T, mn, dv, map_order, I);
   for (int d = 0; d < 3; ++d) {
      SweepCell s;
      float di = (float)I[4 * d + 1], dj = (float)I[4 * d + 2], dk = (float)I[4 * d + 3];
      if (d == 0) { const float t = di; di = dk; dk = t; }
      if (d == 1) { const float t = dj; dj = dk; dk = t; }
      s.intersection = (float)I[4 * d];
      s.di = di;
      s.dj = dj;
      s.dk = dk;
      s.threshold = threshold;
      s.pad = 0;
      sweep3[(size_t)d * n_cells + c] = s;
   }
}

// ---------------------------------------------------------------------------
cudaError_t launch_moments(const uint32_t* gids, const uint32_t* src_index, const float* data, const CellSlot* slots,
                           double* moments,
                           const MeshDev& mesh, const double vmin[3], const double bs[3], const double dv[3],
                           double mass, double charge, bool second, uint32_t n_cells, cudaStream_t stream) {
   if (n_cells == 0) return cudaSuccess;
   moments_kernel<<<n_cells, MOM_THREADS, 0, stream>>>(gids, src_index, data, slots, moments, mesh, vmin[0], vmin[1], vmin[2],
                                                       bs[0], bs[1], bs[2], dv[0], dv[1], dv[2], mass, charge,
                                                       second ? 1 : 0);
   return cudaGetLastError();
}

cudaError_t launch_geometry(const CellAccelInputs* in, const double* moments, double* isect12, SweepCell* sweep3,
                            uint32_t n_cells, double q, double m, double hall_min_rhoq, int ohm_gradpe, double mu0,
                            const double vmin[3], const double dv[3], uint32_t map_order, float threshold,
                            cudaStream_t stream) {
   if (n_cells == 0) return cudaSuccess;
   geometry_kernel<<<(n_cells + 127) / 128, 128, 0, stream>>>(in, moments, isect12, sweep3, n_cells, q, m,
                                                             hall_min_rhoq, ohm_gradpe, mu0, vmin[0], vmin[1],
                                                             vmin[2], dv[0], dv[1], dv[2], map_order, threshold);
   return cudaGetLastError();
}

}  // namespace vlgpu
