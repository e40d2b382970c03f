// Initial phase-space densities on the device: the Maxwellian and
// tri-Maxwellian of projects/project.h:45-73 sampled at the cell centres of
// every candidate block (Project::setVelocitySpace / fillPhaseSpace,
// projects/project.cpp:179-260), written as the batch's block lists; the first
// block adjustment (grid.cpp:289) then prunes them.
#include <cstdint>

#include "batch_internal.cuh"

namespace vlgpu {

// FillCell (batch_internal.cuh): one cell's distribution -- density,
// temperatures along the rows of `frame` (isotropic: the identity and three
// equal temperatures), bulk velocity -- and its candidate block box [lo, hi]
// with the list row of its first candidate.

constexpr int FILL_THREADS = 256;
constexpr double K_B_D = 1.3806503e-23;  // physicalconstants::K_B (common.h:561)

__device__ __forceinline__ double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double da(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsb(double a, double b) { return __dsub_rn(a, b); }

// One CTA per cell: every (candidate block, cell) element of its box.
__global__ void __launch_bounds__(FILL_THREADS) fill_kernel(const FillCell* __restrict__ cells, MeshDev mesh,
                                                            double vmin0, double vmin1, double vmin2, double bs0,
                                                            double bs1, double bs2, double dv0, double dv1,
                                                            double dv2, double mass, uint32_t* __restrict__ gids,
                                                            float* __restrict__ data, CellSlot* __restrict__ slots) {
   const FillCell c = cells[blockIdx.x];
   const int nx = c.hi[0] - c.lo[0] + 1, ny = c.hi[1] - c.lo[1] + 1, nz = c.hi[2] - c.lo[2] + 1;
   const uint32_t nblk = (nx > 0 && ny > 0 && nz > 0) ? (uint32_t)(nx * ny * nz) : 0u;
   if (threadIdx.x == 0) slots[blockIdx.x] = CellSlot{c.row, nblk};
   const double pi = 3.14159265358979323846;
   // the prefactors, in the order the Maxwellian helpers of the projects evaluate them
   double pre, den;
   if (c.isotropic) {
      pre = dm(c.n, pow(mass / dm(dm(dm(2.0, pi), K_B_D), c.T[0]), 1.5));
      den = dm(dm(2.0, K_B_D), c.T[0]);
   } else {
      pre = dm(c.n, pow(mass / dm(dm(2.0, pi), K_B_D), 1.5));
      den = dm(2.0, K_B_D);
   }
   const double inv_sqrtT = c.isotropic ? 1.0 : sqrt(dm(dm(c.T[0], c.T[1]), c.T[2]));
   for (uint64_t e = threadIdx.x; e < (uint64_t)nblk * WID3; e += blockDim.x) {
      const uint32_t q = (uint32_t)(e >> 6);
      const int cc = (int)(e & 63);
      const int bi = c.lo[0] + (int)(q % (uint32_t)nx);
      const int bj = c.lo[1] + (int)((q / (uint32_t)nx) % (uint32_t)ny);
      const int bk = c.lo[2] + (int)(q / (uint32_t)(nx * ny));
      const int ci = cc & 3, cj = (cc >> 2) & 3, ck = cc >> 4;
      const double vx = da(da(vmin0, dm((double)bi, bs0)), dm(ci + 0.5, dv0));
      const double vy = da(da(vmin1, dm((double)bj, bs1)), dm(cj + 0.5, dv1));
      const double vz = da(da(vmin2, dm((double)bk, bs2)), dm(ck + 0.5, dv2));
      const double ux = dsb(vx, c.V[0]), uy = dsb(vy, c.V[1]), uz = dsb(vz, c.V[2]);
      double f;
      if (c.isotropic) {
         const double s = da(da(dm(ux, ux), dm(uy, uy)), dm(uz, uz));
         f = dm(pre, exp(dm(-mass, s) / den));
      } else {
         const double* R = c.frame;
         const double a = da(da(dm(R[0], ux), dm(R[1], uy)), dm(R[2], uz));
         const double b = da(da(dm(R[3], ux), dm(R[4], uy)), dm(R[5], uz));
         const double d = da(da(dm(R[6], ux), dm(R[7], uy)), dm(R[8], uz));
         const double s = da(da(dm(a, a) / c.T[0], dm(b, b) / c.T[1]), dm(d, d) / c.T[2]);
         f = dm(pre, exp(dm(-mass, s) / den)) / inv_sqrtT;
      }
      data[((size_t)c.row + q) * WID3 + cc] = (float)f;
      if (cc == 0) gids[c.row + q] = (uint32_t)bi + mesh.len[0] * ((uint32_t)bj + mesh.len[1] * (uint32_t)bk);
   }
}

cudaError_t launch_fill(const FillCell* cells, uint32_t n_cells, const MeshDev& mesh, const double vmin[3],
                        const double bs[3], const double dv[3], double mass, uint32_t* gids, float* data,
                        CellSlot* slots, cudaStream_t stream) {
   if (n_cells == 0) return cudaSuccess;
   fill_kernel<<<n_cells, FILL_THREADS, 0, stream>>>(cells, mesh, vmin[0], vmin[1], vmin[2], bs[0], bs[1], bs[2],
                                                     dv[0], dv[1], dv[2], mass, gids, data, slots);
   return cudaGetLastError();
}

}  // namespace vlgpu
