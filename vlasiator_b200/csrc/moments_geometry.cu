// Velocity moments (FP64, compensated) and the per-cell FP64 acceleration
// geometry, for sm_100a.
//
// moments_parts_kernel: every cell's blocks in up to 64 equal parts, each
// part summed by one warp (half a warp per velocity block, one float4 x-row
// of four cells per lane) with FP64 arithmetic, the parts of a cell added in
// part order with compensated sums by whichever warp finishes the cell's last
// part.  The sums are those of blockVelocityFirstMoments /
// blockVelocitySecondMoments (vlasovsolver/arch_moments.h:83-155) and the
// per-cell bookkeeping of calculateMoments_V
// (vlasovsolver/arch_moments.cpp:342-499); the pressure tensor comes from
// velocities taken relative to an earlier bulk velocity (see the kernel).
//
// geometry_kernel: one thread per cell builds the gyration transform and the
// three intersection sets in FP64 (geometry.cuh) and converts them into the
// Realf sweep parameters of the three sweeps.
#include <cstdint>

#include "geometry.cuh"
#include "moments_record.cuh"
#include "vlgpu_common.cuh"

namespace vlgpu {

// Each cell's blocks are split into equal parts of at least 32 blocks (at
// most MOM_PARTS_PER_CELL parts); a warp takes (part, cell) items in a fixed
// grid-stride order (consecutive items are the same part of consecutive
// cells, so the work of large and small cells interleaves), sums its part
// with FP64 arithmetic per lane, adds the lanes' sums in lane order, and
// stores the part's sums.  Per lane and block the four cells of a row enter
// as the row's sums of f, i f and i^2 f (i = 0..3), combined with the row's
// first cell centre.  The last
// part of a cell to finish (a per-cell counter) adds the cell's parts in part
// order with compensated sums and writes the record, so the result does not
// depend on which warp ran which part.  Half a warp reads one velocity block,
// each lane one x-row of four cells as a float4 (i = 0..3 at j = sub & 3,
// k = sub >> 2), two blocks per half-warp in flight.
//
// The sums are those of blockVelocityFirstMoments / blockVelocitySecondMoments
// (vlasovsolver/arch_moments.h:83-155) and the record that of
// calculateMoments_V (vlasovsolver/arch_moments.cpp:342-499).  With velocities
// taken relative to a reference velocity U (u = v - U):
//   S0 = sum f, S_a = sum f u_a, S_ab = sum f u_a u_b,
//   n V_a = (S_a + U_a S0) dv^3,  P_ab = m dv^3 (S_ab - S_a S_b / S0).
// With U close to the bulk velocity nothing cancels, and the result equals the
// reference's two-pass sums (first V, then f (v-V)(v-V)) up to FP64 rounding.
//
constexpr int MOM_THREADS = 256;

// Parts of a cell with `count` blocks: enough that a part has at least
// MOM_MIN_PART blocks, at most MOM_PARTS_PER_CELL.
constexpr uint32_t MOM_MIN_PART = 256;
constexpr uint32_t MOM_TILE = 256;  // blocks of a part staged at a time
__device__ __forceinline__ uint32_t moment_parts(uint32_t count) {
   const uint32_t p = (count + MOM_MIN_PART - 1) / MOM_MIN_PART;
   return p < (uint32_t)MOM_PARTS_PER_CELL ? p : (uint32_t)MOM_PARTS_PER_CELL;
}


template <int MODE>
__global__ void __launch_bounds__(MOM_THREADS, 2) moments_parts_kernel(
   const uint32_t* __restrict__ gids, const uint32_t* __restrict__ src_index, const float* __restrict__ data,
   const CellSlot* __restrict__ slots, double* moments, double* pivot, const double* shift,
   double* __restrict__ part_sums, uint32_t* __restrict__ done, MeshDev mesh, double vmin0, double vmin1,
   double vmin2, double bs0, double bs1, double bs2, double dv0, double dv1, double dv2, double mass, double charge,
   uint32_t n_cells) {
   constexpr bool SECOND = MODE != MOM_FIRST;
   constexpr int NS = SECOND ? 10 : 4;
   __shared__ double sh[MOM_THREADS / 32][NS][33];  // a warp's lane sums, one row per sum (padded)
   __shared__ uint32_t sg[MOM_THREADS / 32][MOM_TILE], si[MOM_THREADS / 32][MOM_TILE];  // a tile's block IDs, rows
   const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
   const int half = lane >> 4, sub = lane & 15;
   const int j = sub & 3, k = sub >> 2;
   const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const uint32_t n_warps = (gridDim.x * blockDim.x) >> 5;
   const uint32_t n_items = n_cells * (uint32_t)MOM_PARTS_PER_CELL;
   const double dv0s = dv0 * dv0;
   for (uint32_t it = warp; it < n_items; it += n_warps) {
      const uint32_t part = it / n_cells, cell = it - part * n_cells;
      const CellSlot s = slots[cell];
      const uint32_t parts = moment_parts(s.count);
      if (parts == 0) {
         // a cell without blocks: a zero record (and pivot)
         if (part == 0 && lane < MOM_COUNT) {
            moments[(size_t)cell * MOM_COUNT + lane] = 0.0;
            if (MODE == MOM_BOTH) pivot[(size_t)cell * MOM_COUNT + lane] = 0.0;
         }
         continue;
      }
      if (part >= parts) continue;
      const uint32_t b0 = (uint32_t)(((uint64_t)s.count * part) / parts);
      const uint32_t b1 = (uint32_t)(((uint64_t)s.count * (part + 1)) / parts);
      // the reference velocity: the pivot's (MOM_BOTH) or the shift record's (MOM_SECOND)
      double U0 = 0.0, U1 = 0.0, U2 = 0.0;
      if (MODE == MOM_BOTH) {
         const double* pv = pivot + (size_t)cell * MOM_COUNT;
         U0 = pv[MOM_VX]; U1 = pv[MOM_VY]; U2 = pv[MOM_VZ];
      } else if (MODE == MOM_SECOND) {
         const double* sh_rec = shift + (size_t)cell * MOM_COUNT;
         U0 = sh_rec[MOM_VX]; U1 = sh_rec[MOM_VY]; U2 = sh_rec[MOM_VZ];
      }
      // the first sums are about F (0, or U in MOM_SECOND); a lane's row of
      // four cells starts at the cell centre x0 = corner + dv0/2 - F0, the
      // others follow at dv0 steps
      const double F0 = (MODE == MOM_SECOND) ? U0 : 0.0, F1 = (MODE == MOM_SECOND) ? U1 : 0.0;
      const double F2 = (MODE == MOM_SECOND) ? U2 : 0.0;
      const double ox = 0.5 * dv0 - F0, oy = (j + 0.5) * dv1 - F1, oz = (k + 0.5) * dv2 - F2;
      double t[NS];
#pragma unroll
      for (int q = 0; q < NS; ++q) t[q] = 0.0;
      // tiles of the part: the block IDs and data rows are staged in shared
      // memory (coalesced), then half-warp h reads blocks h, h + 2, h + 4,
      // h + 6 of every eight, all four loads in flight at once
      for (uint32_t t0 = b0; t0 < b1; t0 += MOM_TILE) {
         const uint32_t n = (b1 - t0 < MOM_TILE) ? b1 - t0 : MOM_TILE;
         for (uint32_t q = lane; q < n; q += 32) {
            sg[wl][q] = __ldg(gids + s.off + t0 + q);
            si[wl][q] = src_index ? __ldg(src_index + s.off + t0 + q) : s.off + t0 + q;
         }
         __syncwarp();
         // rows of blocks q0 + 2u (u = 0..3) of this half-warp, the next four
         // prefetched while these are summed
         auto load4 = [&](uint32_t q0, float4* f) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
               const uint32_t q = q0 + 2 * u;
               f[u] = make_float4(0.f, 0.f, 0.f, 0.f);
               if (q < n) {
                  const uint32_t idx = si[wl][q];
                  if (idx != 0xffffffffu)  // an added block holds zeros
                     f[u] = __ldg(reinterpret_cast<const float4*>(data + (size_t)idx * WID3) + sub);
               }
            }
         };
         float4 cur[4], nxt[4];
         load4(half, cur);
         for (uint32_t q0 = half; q0 < n; q0 += 8) {
            load4(q0 + 8, nxt);
#pragma unroll
            for (int u = 0; u < 4; ++u) {
               uint32_t bi, bj, bk;
               block_xyz(mesh, sg[wl][(q0 + 2 * u < n) ? q0 + 2 * u : 0], bi, bj, bk);
               // the row's sums of f, i f and i^2 f (i = 0..3 along x)
               const double d0 = cur[u].x, d1 = cur[u].y, d2 = cur[u].z, d3 = cur[u].w;
               const double s0 = (d0 + d1) + (d2 + d3);
               const double s1 = fma(3.0, d3, fma(2.0, d2, d1));
               const double s2 = fma(9.0, d3, fma(4.0, d2, d1));
               const double x0 = (vmin0 + bi * bs0) + ox;
               const double uy = (vmin1 + bj * bs1) + oy;
               const double uz = (vmin2 + bk * bs2) + oz;
               const double ds1 = dv0 * s1;
               const double sfx = fma(x0, s0, ds1);  // sum f x over the row
               t[0] += s0;
               t[1] += sfx;
               t[2] = fma(s0, uy, t[2]);
               t[3] = fma(s0, uz, t[3]);
               if constexpr (MODE == MOM_SECOND) {
                  // sum f x^2 = x0^2 s0 + 2 x0 dv0 s1 + dv0^2 s2
                  t[4] += fma(x0, fma(x0, s0, 2.0 * ds1), dv0s * s2);
                  const double s0y = s0 * uy;
                  t[5] = fma(s0y, uy, t[5]);
                  t[6] = fma(s0 * uz, uz, t[6]);
                  t[7] = fma(s0y, uz, t[7]);
                  t[8] = fma(sfx, uz, t[8]);
                  t[9] = fma(sfx, uy, t[9]);
               }
               if constexpr (MODE == MOM_BOTH) {
                  // the same row relative to U (the first sums were about 0)
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
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) cur[u] = nxt[u];
         }
         __syncwarp();
      }
      // the part's sums: the warp's lane sums added in lane order by lanes 0..NS-1
#pragma unroll
      for (int q = 0; q < NS; ++q) sh[wl][q][lane] = t[q];
      __syncwarp();
      double* ps = part_sums + ((size_t)cell * MOM_PARTS_PER_CELL + part) * MOM_SUMS_PER_PART;
      if (lane < NS) {
         double v = 0.0;
         for (int l = 0; l < 32; ++l) v += sh[wl][lane][l];
         ps[lane] = v;
      }
      __syncwarp();
      __threadfence();
      uint32_t prev = 0;
      if (lane == 0) prev = atomicAdd(&done[cell], 1u);
      prev = __shfl_sync(0xffffffffu, prev, 0);
      if (prev + 1 != parts) continue;
      // the cell's last part: add all parts in part order
      __threadfence();
      double S = 0.0;
      if (lane < NS) {
         double sum = 0.0, comp = 0.0;
         const double* base = part_sums + (size_t)cell * MOM_PARTS_PER_CELL * MOM_SUMS_PER_PART + lane;
         for (uint32_t p = 0; p < parts; ++p) {
            const double y = __ldcg(base + (size_t)p * MOM_SUMS_PER_PART) - comp;
            const double tt = sum + y;
            comp = (tt - sum) - y;
            sum = tt;
         }
         S = sum - comp;
      }
      double Sv[NS];
#pragma unroll
      for (int q = 0; q < NS; ++q) Sv[q] = __shfl_sync(0xffffffffu, S, q);
      if (lane == 0) {
         moments_record<MODE>(Sv, F0, F1, F2, U0, U1, U2, dv0, dv1, dv2, mass, charge,
                              moments + (size_t)cell * MOM_COUNT,
                              MODE == MOM_BOTH ? pivot + (size_t)cell * MOM_COUNT : nullptr);
         done[cell] = 0;  // ready for the next pass
      }
   }
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
int moments_blocks_per_sm() {
   int n = 0;
   cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, moments_parts_kernel<MOM_BOTH>, MOM_THREADS, 0);
   return n > 0 ? n : 1;
}

cudaError_t launch_moments(const uint32_t* gids, const uint32_t* src_index, const float* data, const CellSlot* slots,
                           double* moments, const double* shift, const MeshDev& mesh, const double vmin[3],
                           const double bs[3], const double dv[3], double mass, double charge, bool second,
                           uint32_t n_cells, double* part_sums, uint32_t* done, int grid, cudaStream_t stream) {
   if (n_cells == 0) return cudaSuccess;
   if (!shift) shift = moments;
   if (second)
      moments_parts_kernel<MOM_SECOND><<<grid, MOM_THREADS, 0, stream>>>(
         gids, src_index, data, slots, moments, nullptr, shift, part_sums, done, mesh, vmin[0], vmin[1], vmin[2],
         bs[0], bs[1], bs[2], dv[0], dv[1], dv[2], mass, charge, n_cells);
   else
      moments_parts_kernel<MOM_FIRST><<<grid, MOM_THREADS, 0, stream>>>(
         gids, src_index, data, slots, moments, nullptr, shift, part_sums, done, mesh, vmin[0], vmin[1], vmin[2],
         bs[0], bs[1], bs[2], dv[0], dv[1], dv[2], mass, charge, n_cells);
   return cudaGetLastError();
}

cudaError_t launch_moments_both(const uint32_t* gids, const uint32_t* src_index, const float* data,
                                const CellSlot* slots, double* pivot, double* moments, const MeshDev& mesh,
                                const double vmin[3], const double bs[3], const double dv[3], double mass,
                                double charge, uint32_t n_cells, double* part_sums, uint32_t* done, int grid,
                                cudaStream_t stream) {
   if (n_cells == 0) return cudaSuccess;
   moments_parts_kernel<MOM_BOTH><<<grid, MOM_THREADS, 0, stream>>>(
      gids, src_index, data, slots, moments, pivot, nullptr, part_sums, done, mesh, vmin[0], vmin[1], vmin[2], bs[0],
      bs[1], bs[2], dv[0], dv[1], dv[2], mass, charge, n_cells);
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
