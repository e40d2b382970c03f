// Velocity moments (FP64, Kahan-compensated) and the per-cell FP64
// acceleration geometry, for sm_100a.
//
// moments_kernel: one CTA per cell, one pass over the cell's data.  Sixteen
// threads share a velocity block, each reading one x-row of four cells as a
// float4, with several blocks in flight per thread group; per-thread partial
// sums are Kahan-compensated doubles, merged across the CTA with error-free
// (TwoSum) additions.  The sums are those of blockVelocityFirstMoments /
// blockVelocitySecondMoments (vlasovsolver/arch_moments.h:83-155) and the
// per-cell bookkeeping of calculateMoments_V
// (vlasovsolver/arch_moments.cpp:342-499); the pressure tensor comes from
// velocities taken relative to the previous bulk velocity (see the kernel).
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
constexpr int MOM_GROUPS = MOM_THREADS / 16;  // 16 threads per velocity block
constexpr int MOM_MAXSUMS = 10;

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

// One CTA per cell; 16 threads per velocity block, each owning one x-row of
// four cells (a float4: i = 0..3 at j = sub & 3, k = sub >> 2), and every
// thread group keeps MOM_UNROLL blocks in flight.  With SECOND, velocities
// are taken relative to a reference velocity U (a bulk velocity of an
// earlier VDF of the cell: the acceleration step's pivot), so one pass over
// the data gives both the first moments and the central second moments:
//   S0 = sum f, S_a = sum f u_a, S_ab = sum f u_a u_b   (u = v - U)
//   n V_a = (S_a + U_a S0) dv^3,  P_ab = m dv^3 (S_ab - S_a S_b / S0).
// With U close to V the correction term is small, so nothing cancels; the
// result equals the reference's two-pass sums (first V, then f (v-V)(v-V))
// up to FP64 rounding.  Without SECOND, U = 0, so the first moments depend
// on the data alone.
//
// moments_pass is one such pass of a CTA over one cell's blocks; thread 0
// writes the cell's record `out`.
//
// MODE MOM_BOTH does the work of a first-moments pass and a second-moments
// pass in one read: the first sums with U = 0 (the same arithmetic as
// MOM_FIRST, so the first moments are identical) and the second sums about
// the U given, whose first sums T_a = S_a - U_a S0 follow from the former;
// the cancellation in T_a costs about eps (U / v_th)^2 of P relative, far
// below the tolerance of any use, and vanishes as U approaches V.  It writes
// the first moments to `out1` (pressure zero, as MOM_FIRST) and everything
// to `out`.
constexpr int MOM_FIRST = 0, MOM_SECOND = 1, MOM_BOTH = 2;

template <int MODE>
__device__ __forceinline__ void moments_pass(const uint32_t* __restrict__ gids, const uint32_t* __restrict__ src_index,
                                             const float* __restrict__ data, const CellSlot s, double* out,
                                             const MeshDev& mesh, double vmin0, double vmin1, double vmin2, double bs0,
                                             double bs1, double bs2, double dv0, double dv1, double dv2, double mass,
                                             double charge, double U0, double U1, double U2, double* sh_hi,
                                             double* sh_lo, double* out1 = nullptr) {
   constexpr bool SECOND = MODE != MOM_FIRST;
   constexpr int NS = SECOND ? 10 : 4;
   const int sub = threadIdx.x & 15, grp = threadIdx.x >> 4;
   const int j = sub & 3, k = sub >> 2;
   // velocity offsets of the first sums (U = 0 in MOM_BOTH) and of the second
   const double F0 = (MODE == MOM_BOTH) ? 0.0 : U0, F1 = (MODE == MOM_BOTH) ? 0.0 : U1;
   const double F2 = (MODE == MOM_BOTH) ? 0.0 : U2;
   const double cy = (j + 0.5) * dv1 - F1, cz = (k + 0.5) * dv2 - F2;
   const double cx0 = 0.5 * dv0 - F0, cx1 = 1.5 * dv0 - F0, cx2 = 2.5 * dv0 - F0, cx3 = 3.5 * dv0 - F0;
   const double sy = (j + 0.5) * dv1 - U1, sz = (k + 0.5) * dv2 - U2;
   const double sx0 = 0.5 * dv0 - U0, sx1 = 1.5 * dv0 - U0, sx2 = 2.5 * dv0 - U0, sx3 = 3.5 * dv0 - U0;
   Kahan acc[NS];
   constexpr int MOM_UNROLL = (MODE == MOM_FIRST) ? 8 : (MODE == MOM_SECOND ? 4 : 2);  // blocks in flight per group
   constexpr uint32_t STEP = MOM_GROUPS * MOM_UNROLL;
   // block IDs and data indices of a batch; the next batch's are loaded while
   // the current batch's data is in flight, so a batch waits on one round
   // trip to memory, not on the index lookup before it
   uint32_t g[MOM_UNROLL], idx[MOM_UNROLL];
   auto fetch = [&](uint32_t b0, uint32_t* gg, uint32_t* ii) {
#pragma unroll
      for (int u = 0; u < MOM_UNROLL; ++u) {
         const uint32_t b = b0 + u * MOM_GROUPS;
         gg[u] = (b < s.count) ? __ldg(gids + s.off + b) : 0u;
         ii[u] = (b < s.count) ? (src_index ? __ldg(src_index + s.off + b) : s.off + b) : 0xffffffffu;
      }
   };
   fetch(grp, g, idx);
   // per-thread sums of a batch, added to the compensated sums once per
   // batch; in MOM_BOTH the first sums keep MOM_FIRST's batches of 8 blocks
   // (four of its batches of 2, same blocks in the same order), so that its
   // first moments are bit-identical to a MOM_FIRST pass
   double t[NS];
#pragma unroll
   for (int q = 0; q < NS; ++q) t[q] = 0.0;
   int vb = 0;
   for (uint32_t b0 = grp; b0 < s.count; b0 += STEP) {
      float4 f4[MOM_UNROLL];
#pragma unroll
      for (int u = 0; u < MOM_UNROLL; ++u) {
         f4[u] = make_float4(0.f, 0.f, 0.f, 0.f);
         if (idx[u] != 0xffffffffu)  // an added block holds zeros
            f4[u] = __ldg(reinterpret_cast<const float4*>(data + (size_t)idx[u] * WID3) + sub);
      }
      uint32_t g_next[MOM_UNROLL], idx_next[MOM_UNROLL];
      fetch(b0 + STEP, g_next, idx_next);
#pragma unroll
      for (int u = 0; u < MOM_UNROLL; ++u) {
         uint32_t bi, bj, bk;
         block_xyz(mesh, g[u], bi, bj, bk);
         const double bx = vmin0 + bi * bs0;
         const double uy = (vmin1 + bj * bs1) + cy;
         const double uz = (vmin2 + bk * bs2) + cz;
         const double x0 = bx + cx0, x1 = bx + cx1, x2 = bx + cx2, x3 = bx + cx3;
         const double f0 = f4[u].x, f1 = f4[u].y, f2 = f4[u].z, f3 = f4[u].w;
         const double sf = (f0 + f1) + (f2 + f3);
         const double fx0 = f0 * x0, fx1 = f1 * x1, fx2 = f2 * x2, fx3 = f3 * x3;
         const double sfx = (fx0 + fx1) + (fx2 + fx3);
         t[0] += sf;
         t[1] += sfx;
         t[2] += sf * uy;
         t[3] += sf * uz;
         if constexpr (MODE == MOM_SECOND) {
            t[4] += (fx0 * x0 + fx1 * x1) + (fx2 * x2 + fx3 * x3);
            t[5] += sf * uy * uy;
            t[6] += sf * uz * uz;
            t[7] += sf * uy * uz;
            t[8] += sfx * uz;
            t[9] += sfx * uy;
         }
         if constexpr (MODE == MOM_BOTH) {
            const double vy = (vmin1 + bj * bs1) + sy, vz = (vmin2 + bk * bs2) + sz;
            const double y0 = bx + sx0, y1 = bx + sx1, y2 = bx + sx2, y3 = bx + sx3;
            const double fy0 = f0 * y0, fy1 = f1 * y1, fy2 = f2 * y2, fy3 = f3 * y3;
            const double sfy = (fy0 + fy1) + (fy2 + fy3);
            t[4] += (fy0 * y0 + fy1 * y1) + (fy2 * y2 + fy3 * y3);
            t[5] += sf * vy * vy;
            t[6] += sf * vz * vz;
            t[7] += sf * vy * vz;
            t[8] += sfy * vz;
            t[9] += sfy * vy;
         }
      }
      if constexpr (MODE == MOM_BOTH) {
#pragma unroll
         for (int q = 4; q < NS; ++q) {
            acc[q].add(t[q]);
            t[q] = 0.0;
         }
         if (++vb == 4) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
               acc[q].add(t[q]);
               t[q] = 0.0;
            }
            vb = 0;
         }
      } else {
#pragma unroll
         for (int q = 0; q < NS; ++q) {
            acc[q].add(t[q]);
            t[q] = 0.0;
         }
      }
#pragma unroll
      for (int u = 0; u < MOM_UNROLL; ++u) {
         g[u] = g_next[u];
         idx[u] = idx_next[u];
      }
   }
   if (MODE == MOM_BOTH && vb) {
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q].add(t[q]);
   }
   double hi[NS], lo[NS];
#pragma unroll
   for (int q = 0; q < NS; ++q) {
      hi[q] = acc[q].s;
      lo[q] = -acc[q].c;
   }
   cta_reduce<NS>(hi, lo, sh_hi, sh_lo);
   if (threadIdx.x != 0) return;
   double S[NS];
#pragma unroll
   for (int q = 0; q < NS; ++q) S[q] = hi[q] + lo[q];
   const double DV3 = dv0 * dv1 * dv2;
   const double a0 = S[0] * DV3;
   const double a1 = (S[1] + F0 * S[0]) * DV3, a2 = (S[2] + F1 * S[0]) * DV3, a3 = (S[3] + F2 * S[0]) * DV3;
   out[MOM_N] = a0;
   out[MOM_NVX] = a1;
   out[MOM_NVY] = a2;
   out[MOM_NVZ] = a3;
   const double rhom = a0 * mass;
   out[MOM_RHOM] = rhom;
   out[MOM_VX] = (rhom != 0.0) ? (a1 * mass) / rhom : 0.0;
   out[MOM_VY] = (rhom != 0.0) ? (a2 * mass) / rhom : 0.0;
   out[MOM_VZ] = (rhom != 0.0) ? (a3 * mass) / rhom : 0.0;
   out[MOM_RHOQ] = a0 * charge;
   out[MOM_MASS] = S[0];
   double P[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
   if constexpr (SECOND) {
      if (S[0] != 0.0) {
         // first sums about U (those of MOM_BOTH were taken about 0)
         const double T1 = (MODE == MOM_BOTH) ? S[1] - U0 * S[0] : S[1];
         const double T2 = (MODE == MOM_BOTH) ? S[2] - U1 * S[0] : S[2];
         const double T3 = (MODE == MOM_BOTH) ? S[3] - U2 * S[0] : S[3];
         const double m1 = T1 / S[0], m2 = T2 / S[0], m3 = T3 / S[0];
         const double pre = mass * DV3;
         P[0] = pre * (S[4] - T1 * m1);
         P[1] = pre * (S[5] - T2 * m2);
         P[2] = pre * (S[6] - T3 * m3);
         P[3] = pre * (S[7] - T2 * m3);
         P[4] = pre * (S[8] - T1 * m3);
         P[5] = pre * (S[9] - T1 * m2);
      }
   }
   for (int q = 0; q < 6; ++q) out[MOM_P11 + q] = P[q];
   if (MODE == MOM_BOTH && out1) {
      for (int q = 0; q < MOM_COUNT; ++q) out1[q] = (q >= MOM_P11 && q < MOM_P11 + 6) ? 0.0 : out[q];
   }
}

// With SECOND the reference velocity U is the bulk velocity in the cell's
// record of `shift`.
template <bool SECOND>
__global__ void __launch_bounds__(MOM_THREADS, 2) moments_kernel(
   const uint32_t* __restrict__ gids, const uint32_t* __restrict__ src_index, const float* __restrict__ data,
   const CellSlot* __restrict__ slots, double* moments, const double* shift, MeshDev mesh, double vmin0,
   double vmin1, double vmin2, double bs0, double bs1, double bs2, double dv0, double dv1, double dv2, double mass,
   double charge) {
   __shared__ double sh_hi[(MOM_THREADS / 32) * MOM_MAXSUMS];
   __shared__ double sh_lo[(MOM_THREADS / 32) * MOM_MAXSUMS];
   const uint32_t cell = blockIdx.x;
   double* out = moments + (size_t)cell * MOM_COUNT;
   const double* sh = shift + (size_t)cell * MOM_COUNT;
   const double U0 = SECOND ? sh[MOM_VX] : 0.0, U1 = SECOND ? sh[MOM_VY] : 0.0, U2 = SECOND ? sh[MOM_VZ] : 0.0;
   moments_pass<SECOND ? MOM_SECOND : MOM_FIRST>(gids, src_index, data, slots[cell], out, mesh, vmin0, vmin1, vmin2,
                                                 bs0, bs1, bs2, dv0, dv1, dv2, mass, charge, U0, U1, U2, sh_hi, sh_lo);
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
      s.flags = (a.dt == 0.0) ? SWEEP_PASS : 0u;
      sweep3[(size_t)d * n_cells + c] = s;
   }
}

// ---------------------------------------------------------------------------
// Time-step limits per cell: the r-space limit of reduce_vlasov_dt
// (vlasovsolver/arch_dt.cpp:34-97), min over blocks and over the first and
// last cell of the block of min(dx/|vx|, dy/|vy|, dz/|vz|) at those cells'
// centres (+1000*DBL_MIN), and the v-space limit of updateAccelerationMaxdt
// (cpu_acc_transform.cpp:41-55), |gyroperiod| * max_rotation/360.
// ---------------------------------------------------------------------------
constexpr int DT_THREADS = 128;

__global__ void __launch_bounds__(DT_THREADS) max_dt_kernel(
   const uint32_t* __restrict__ gids, const CellSlot* __restrict__ slots, const CellAccelInputs* __restrict__ in,
   MeshDev mesh, double vmin0, double vmin1, double vmin2, double bs0, double bs1, double bs2, double dv0, double dv1,
   double dv2, double dx, double dy, double dz, double q, double m, double max_rotation_deg, double* __restrict__ r_dt,
   double* __restrict__ v_dt) {
   __shared__ double s_min[DT_THREADS / 32];
   const uint32_t cell = blockIdx.x;
   const CellSlot s = slots[cell];
   const double EPS = 2.2250738585072014e-308 * 1000;  // numeric_limits<Real>::min() * 1000
   double t = 1.7976931348623157e308;
   for (uint32_t b = threadIdx.x; b < s.count; b += blockDim.x) {
      const uint32_t g = gids[s.off + b];
      const uint32_t bi = g % mesh.len[0], bj = (g / mesh.len[0]) % mesh.len[1], bk = g / (mesh.len[0] * mesh.len[1]);
      const double cx = vmin0 + bi * bs0, cy = vmin1 + bj * bs1, cz = vmin2 + bk * bs2;
      for (int i = 0; i < WID; i += WID - 1) {
         const double Vx = cx + (i + 0.5) * dv0 + EPS;
         const double Vy = cy + (i + 0.5) * dv1 + EPS;
         const double Vz = cz + (i + 0.5) * dv2 + EPS;
         t = fmin(t, fmin(dx / fabs(Vx), fmin(dy / fabs(Vy), dz / fabs(Vz))));
      }
   }
#pragma unroll
   for (int o = 16; o >= 1; o >>= 1) t = fmin(t, __shfl_xor_sync(0xffffffffu, t, o));
   if ((threadIdx.x & 31) == 0) s_min[threadIdx.x >> 5] = t;
   __syncthreads();
   if (threadIdx.x == 0) {
      for (int w = 1; w < DT_THREADS / 32; ++w) t = fmin(t, s_min[w]);
      r_dt[cell] = t;
      const CellAccelInputs a = in[cell];
      const double B_mag = sqrt(a.B[0] * a.B[0] + a.B[1] * a.B[1] + a.B[2] * a.B[2]) + 1e-30;
      const double gyro_period = 2 * M_PI * m / (q * B_mag);
      v_dt[cell] = fabs(gyro_period) * (max_rotation_deg / 360.0);
   }
}

cudaError_t launch_max_dt(const uint32_t* gids, const CellSlot* slots, const CellAccelInputs* in, const MeshDev& mesh,
                          const double vmin[3], const double bs[3], const double dv[3], const double dx[3], double q,
                          double m, double max_rotation_deg, double* r_dt, double* v_dt, uint32_t n_cells,
                          cudaStream_t stream) {
   if (n_cells == 0) return cudaSuccess;
   max_dt_kernel<<<n_cells, DT_THREADS, 0, stream>>>(gids, slots, in, mesh, vmin[0], vmin[1], vmin[2], bs[0], bs[1],
                                                     bs[2], dv[0], dv[1], dv[2], dx[0], dx[1], dx[2], q, m,
                                                     max_rotation_deg, r_dt, v_dt);
   return cudaGetLastError();
}

// ---------------------------------------------------------------------------
cudaError_t launch_moments(const uint32_t* gids, const uint32_t* src_index, const float* data, const CellSlot* slots,
                           double* moments, const double* shift, const MeshDev& mesh, const double vmin[3],
                           const double bs[3], const double dv[3], double mass, double charge, bool second,
                           uint32_t n_cells, cudaStream_t stream) {
   if (n_cells == 0) return cudaSuccess;
   if (!shift) shift = moments;
   if (second)
      moments_kernel<true><<<n_cells, MOM_THREADS, 0, stream>>>(gids, src_index, data, slots, moments, shift, mesh,
                                                               vmin[0], vmin[1], vmin[2], bs[0], bs[1], bs[2], dv[0],
                                                               dv[1], dv[2], mass, charge);
   else
      moments_kernel<false><<<n_cells, MOM_THREADS, 0, stream>>>(gids, src_index, data, slots, moments, shift, mesh,
                                                                vmin[0], vmin[1], vmin[2], bs[0], bs[1], bs[2], dv[0],
                                                                dv[1], dv[2], mass, charge);
   return cudaGetLastError();
}

// MOM_BOTH of every cell: reference velocity U from the cell's record in
// `pivot`, which then receives the first moments of this VDF; the moments
// with pressure go to `moments`.
__global__ void __launch_bounds__(MOM_THREADS, 2) moments_both_kernel(
   const uint32_t* __restrict__ gids, const uint32_t* __restrict__ src_index, const float* __restrict__ data,
   const CellSlot* __restrict__ slots, double* pivot, double* __restrict__ moments, MeshDev mesh, double vmin0,
   double vmin1, double vmin2, double bs0, double bs1, double bs2, double dv0, double dv1, double dv2, double mass,
   double charge) {
   __shared__ double sh_hi[(MOM_THREADS / 32) * MOM_MAXSUMS];
   __shared__ double sh_lo[(MOM_THREADS / 32) * MOM_MAXSUMS];
   const uint32_t cell = blockIdx.x;
   double* pv = pivot + (size_t)cell * MOM_COUNT;
   const double U0 = pv[MOM_VX], U1 = pv[MOM_VY], U2 = pv[MOM_VZ];
   __syncthreads();  // every thread has read U before thread 0 overwrites the record
   moments_pass<MOM_BOTH>(gids, src_index, data, slots[cell], moments + (size_t)cell * MOM_COUNT, mesh, vmin0, vmin1,
                          vmin2, bs0, bs1, bs2, dv0, dv1, dv2, mass, charge, U0, U1, U2, sh_hi, sh_lo, pv);
}

cudaError_t launch_moments_both(const uint32_t* gids, const uint32_t* src_index, const float* data,
                                const CellSlot* slots, double* pivot, double* moments, const MeshDev& mesh,
                                const double vmin[3], const double bs[3], const double dv[3], double mass,
                                double charge, uint32_t n_cells, cudaStream_t stream) {
   if (n_cells == 0) return cudaSuccess;
   moments_both_kernel<<<n_cells, MOM_THREADS, 0, stream>>>(gids, src_index, data, slots, pivot, moments, mesh,
                                                           vmin[0], vmin[1], vmin[2], bs[0], bs[1], bs[2], dv[0],
                                                           dv[1], dv[2], mass, charge);
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
