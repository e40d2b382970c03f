// The per-cell moment record of a batch and how it is formed from FP64 sums
// (shared by the moments kernels and the adjustment, which fuses the "_V"
// moments into its pass over the blocks).
#pragma once
#include <cstdint>

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

// Modes: MOM_FIRST sums the first moments about 0; MOM_SECOND sums everything
// about the U of the `shift` record; MOM_BOTH does both passes' work in one
// read: the first sums about 0 with exactly MOM_FIRST's arithmetic (so the
// first moments, which the next acceleration takes as its pivot, are
// bit-identical to a MOM_FIRST pass) and the second sums about the U of the
// pivot record, whose first sums T_a = S_a - U_a S0 follow from the former;
// the cancellation in T_a costs about eps (U / v_th)^2 of P relative and
// vanishes as U approaches V.  MOM_BOTH writes the full record to `out` and
// the first moments (pressure zero, as MOM_FIRST) to the pivot record.
constexpr int MOM_FIRST = 0, MOM_SECOND = 1, MOM_BOTH = 2;

// The record of a cell from its sums S (about U for the second moments; the
// first sums about F, which is 0 or U).
template <int MODE>
__device__ __forceinline__ void moments_record(const double* S, double F0, double F1, double F2, double U0, double U1,
                                            double U2, double dv0, double dv1, double dv2, double mass, double charge,
                                            double* out, double* out1) {
   constexpr bool SECOND = MODE != MOM_FIRST;
   const double DV3 = dv0 * dv1 * dv2;
   const double a0 = S[0] * DV3;
   const double a1 = (S[1] + F0 * S[0]) * DV3, a2 = (S[2] + F1 * S[0]) * DV3, a3 = (S[3] + F2 * S[0]) * DV3;
   const double rhom = a0 * mass;
   const double first[MOM_P11] = {a0,
                                  a1,
                                  a2,
                                  a3,
                                  rhom,
                                  (rhom != 0.0) ? (a1 * mass) / rhom : 0.0,
                                  (rhom != 0.0) ? (a2 * mass) / rhom : 0.0,
                                  (rhom != 0.0) ? (a3 * mass) / rhom : 0.0,
                                  a0 * charge};
#pragma unroll
   for (int q = 0; q < MOM_P11; ++q) {
      out[q] = first[q];
      if (MODE == MOM_BOTH && out1) out1[q] = first[q];
   }
   out[MOM_MASS] = S[0];
   if (MODE == MOM_BOTH && out1) {
      out1[MOM_MASS] = S[0];
#pragma unroll
      for (int q = 0; q < 6; ++q) out1[MOM_P11 + q] = 0.0;
   }
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
#pragma unroll
   for (int q = 0; q < 6; ++q) out[MOM_P11 + q] = P[q];
}

}  // namespace vlgpu
