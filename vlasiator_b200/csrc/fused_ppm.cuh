// Reconstruction coefficients (PLM, PPM, PQM) and their integrals in plain
// single precision: the fused arithmetic of the acceleration and translation
// remaps.
#pragma once

namespace vlgpu {

// Superbee slope of (l, m, r) on unscaled values: sign(a) * max(min(|a|, 2|b|),
// min(2|a|, |b|)) when a b > 0 (a = r - m, b = m - l), else 0.
__device__ __forceinline__ float superbee_fused(float l, float m, float r) {
   const float a = r - m, b = m - l;
   const bool same = a * b > 0.0f;
   const float aa = fabsf(a), ab = fabsf(b);
   return same ? copysignf(fmaxf(fminf(aa, ab + ab), fminf(aa + aa, ab)), a) : 0.0f;
}

// PLM coefficients (compute_plm_coeff, cpu_1d_plm.hpp:38-49): f = a0 + 2 a1 t.
__device__ __forceinline__ void plm_coeff_fused(float vm1, float v0, float vp1, float a[5]) {
   const float d = superbee_fused(vm1, v0, vp1);
   a[0] = v0 - 0.5f * d;
   a[1] = 0.5f * d;
}

// h8 face value and h7 face derivative of the left face of the cell whose
// stencil is w0..w7 = values k-4 .. k+3 (cpu_face_estimates.hpp:45-79).
__device__ __forceinline__ float h8_value(float w0, float w1, float w2, float w3, float w4, float w5, float w6,
                                          float w7) {
   return (float)(1.0 / 840.0) *
          (533.0f * (w3 + w4) - 139.0f * (w2 + w5) + 29.0f * (w1 + w6) - 3.0f * (w0 + w7));
}
__device__ __forceinline__ float h7_derivative(float w0, float w1, float w2, float w3, float w4, float w5, float w6,
                                               float w7) {
   return (float)(1.0 / 5040.0) *
          (7175.0f * (w4 - w3) - 889.0f * (w5 - w2) + 119.0f * (w6 - w1) - 9.0f * (w7 - w0));
}

// PQM coefficients (compute_pqm_coeff, cpu_1d_pqm.hpp:157-176) from the raw
// h8/h7 faces: the extremum / boundedness / slope filters of
// compute_filtered_face_values_derivatives (cpu_face_estimates.hpp:216-275)
// and the inflexion-point filter filter_pqm_monotonicity (cpu_1d_pqm.hpp:
// 31-156), in single precision.
__device__ __forceinline__ void pqm_coeff_fused(float vm1, float v0, float vp1, float fv_l, float fv_r, float fd_l,
                                                float fd_r, float a[5]) {
   const float slope = superbee_fused(vm1, v0, vp1);
   const float slope_abs = fabsf(slope);
   const float slope_sign = slope > 0.0f ? 1.0f : -1.0f;
   if (slope_abs == 0.0f) {
      fv_r = v0;
      fv_l = v0;
      fd_l = 0.0f;
      fd_r = 0.0f;
   }
   if ((vm1 - fv_l) * (fv_l - v0) < 0.0f || slope_sign * fd_l < 0.0f) {
      fv_l = v0 - slope_sign * 0.5f * slope_abs;
      fd_l = slope_sign * slope_abs;
   }
   if ((vp1 - fv_r) * (fv_r - v0) < 0.0f || slope_sign * fd_r < 0.0f) {
      fv_r = v0 + slope_sign * 0.5f * slope_abs;
      fd_r = slope_sign * slope_abs;
   }
   // second-derivative coefficients (White and Adcroft 2008, eq. 23)
   const float b0 = 60.0f * v0 - 24.0f * fv_r - 36.0f * fv_l + 3.0f * (fd_r - 3.0f * fd_l);
   const float b1 = -360.0f * v0 + 36.0f * fd_l - 24.0f * fd_r + 168.0f * fv_r + 192.0f * fv_l;
   const float b2 = 360.0f * v0 + 30.0f * (fd_r - fd_l) - 180.0f * (fv_l + fv_r);
   const float disc = b1 * b1 - 4.0f * b0 * b2;
   const float sq = disc < 0.0f ? b1 + 200.0f * b2 : sqrtf(disc);
   const float root1 = (-b1 + sq) / (2.0f * b2);
   const float root2 = (-b1 - sq) / (2.0f * b2);
   const float plm_l = 2.0f * (v0 - vm1), plm_r = 2.0f * (vp1 - v0);
   const float ssign = plm_l + plm_r;
   const float c0 = fd_l, c1 = b0, c2 = 0.5f * b1, c3 = b2 * (float)(1.0 / 3.0);
   const float r1s = (root1 >= 0.0f && root1 <= 1.0f) ? c0 + root1 * (c1 + root1 * (c2 + root1 * c3)) : ssign;
   const float r2s = (root2 >= 0.0f && root2 <= 1.0f) ? c0 + root2 * (c1 + root2 * (c2 + root2 * c3)) : ssign;
   if (r1s * ssign < 0.0f || r2s * ssign < 0.0f) {
      const float third = (float)(1.0 / 3.0);
      if (fabsf(plm_l) <= fabsf(plm_r)) {
         // collapse to the left edge (eq. 21), then the PLM-slope checks (eqs. 28, 29)
         fd_l = third * (10.0f * v0 - 2.0f * fv_r - 8.0f * fv_l);
         fd_r = -10.0f * v0 + 6.0f * fv_r + 4.0f * fv_l;
         if (ssign * fd_l < 0.0f) {
            fd_l = 0.0f;
            fv_r = 5.0f * v0 - 4.0f * fv_l;
            fd_r = 20.0f * (v0 - fv_l);
         } else if (ssign * fd_r < 0.0f) {
            fd_r = 0.0f;
            fv_l = 0.5f * (5.0f * v0 - 3.0f * fv_r);
            fd_l = (float)(10.0 / 3.0) * (-v0 + fv_r);
         }
      } else {
         fd_l = 10.0f * v0 - 6.0f * fv_l - 4.0f * fv_r;
         fd_r = third * (-10.0f * v0 + 2.0f * fv_l + 8.0f * fv_r);
         if (ssign * fd_l < 0.0f) {
            fd_l = 0.0f;
            fv_r = 0.5f * (5.0f * v0 - 3.0f * fv_l);
            fd_r = (float)(10.0 / 3.0) * (v0 - fv_l);
         } else if (ssign * fd_r < 0.0f) {
            fd_r = 0.0f;
            fv_l = 5.0f * v0 - 4.0f * fv_r;
            fd_l = 20.0f * (-v0 + fv_r);
         }
      }
   }
   a[0] = fv_l;
   a[1] = 0.5f * fd_l;
   a[2] = 10.0f * v0 - 4.0f * fv_r - 6.0f * fv_l + 0.5f * (fd_r - 3.0f * fd_l);
   a[3] = -15.0f * v0 + 1.5f * fd_l - fd_r + 7.0f * fv_r + 8.0f * fv_l;
   a[4] = 6.0f * v0 + 0.5f * (fd_r - fd_l) - 3.0f * (fv_l + fv_r);
}

// Reconstruction orders of the acceleration remap (the reference's
// ACC_SEMILAG_PLM / _PPM / _PQM).
constexpr int RECON_PLM = 1, RECON_PPM = 2, RECON_PQM = 4;

// Integral of the reconstruction from 0 to u (cpu_acc_map.cpp:585-601),
// Horner form with FMA.
template <int RECON>
__device__ __forceinline__ float recon_integral(float u, const float a[5]) {
   if constexpr (RECON == RECON_PLM) return u * fmaf(u, a[1], a[0]);
   if constexpr (RECON == RECON_PPM) return u * fmaf(u, fmaf(u, a[2], a[1]), a[0]);
   return u * fmaf(u, fmaf(u, fmaf(u, fmaf(u, a[4], a[3]), a[2]), a[1]), a[0]);
}

// The h4 face of uniform cells, (-v_{-2} + 7 v_{-1} + 7 v_0 - v_1) / 12
// (cpu_face_estimates.hpp:160-167), in single precision with FMA.
__device__ __forceinline__ float h4_face_fused(float vm2, float vm1, float v0, float vp1) {
   return fmaf(7.0f, vm1 + v0, -(vm2 + vp1)) * (float)(1.0 / 12.0);
}

// The same face and PPM for two independent cells at once, with the packed
// single-precision operations of sm_100 (__fadd2_rn, __fmul2_rn, __ffma2_rn;
// y - x as fma(x, -1, y), exact before rounding); the limiter's comparisons
// and selections stay per component.
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 p_sub(float2 y, float2 x) { return __ffma2_rn(x, f2(-1.0f), y); }

__device__ __forceinline__ float2 h4_face_x2(float2 vm2, float2 vm1, float2 v0, float2 vp1) {
   return __ffma2_rn(__fadd2_rn(vm1, v0), f2((float)(7.0 / 12.0)),
                     __fmul2_rn(__fadd2_rn(vm2, vp1), f2((float)(-1.0 / 12.0))));
}

// Superbee slope magnitude of one cell (zero at an extremum), the faces
// flattened to v0 where it is zero, and half the signed slope.
__device__ __forceinline__ float half_slope(float a, float b, float v0, float& fl, float& fr) {
   const bool same = a * b > 0.0f;
   const float aa = fabsf(a), ab = fabsf(b);
   const float sl = same ? fmaxf(fminf(aa, ab + ab), fminf(aa + aa, ab)) : 0.0f;
   if (sl == 0.0f) {
      fl = v0;
      fr = v0;
   }
   return copysignf(0.5f * sl, a);
}

// PPM coefficients of two cells at once (cpu_1d_ppm.hpp:35-54 in plain single
// precision: superbee slope, faces outside their cells' values reset to
// v0 -/+ slope/2, Colella-Woodward overshoot corrections): f(t) = a0 + a1 t +
// a2 t^2 on each.
__device__ __forceinline__ void ppm_coeff_x2(float2 vm1, float2 v0, float2 vp1, float2 fl, float2 fr, float2& a0,
                                             float2& a1, float2& a2) {
   const float2 a = p_sub(vp1, v0), b = p_sub(v0, vm1);
   float2 hs;
   hs.x = half_slope(a.x, b.x, v0.x, fl.x, fr.x);
   hs.y = half_slope(a.y, b.y, v0.y, fl.y, fr.y);
   {
      const float2 tl = __fmul2_rn(p_sub(vm1, fl), p_sub(fl, v0));
      const float2 tr = __fmul2_rn(p_sub(vp1, fr), p_sub(fr, v0));
      const float2 nl = p_sub(v0, hs), nr = __fadd2_rn(v0, hs);
      if (tl.x < 0.0f) fl.x = nl.x;
      if (tl.y < 0.0f) fl.y = nl.y;
      if (tr.x < 0.0f) fr.x = nr.x;
      if (tr.y < 0.0f) fr.y = nr.y;
   }
   const float2 sixth = f2((float)(1.0 / 6.0));
   const float2 v3 = __fmul2_rn(v0, f2(3.0f));
   {
      const float2 d = p_sub(fr, fl), e = __ffma2_rn(__fadd2_rn(fl, fr), f2(-0.5f), v0);
      const float2 de = __fmul2_rn(d, e), dd = __fmul2_rn(__fmul2_rn(d, d), sixth);
      const float2 alt = __ffma2_rn(fr, f2(-2.0f), v3);
      if (de.x > dd.x) fl.x = alt.x;
      if (de.y > dd.y) fl.y = alt.y;
   }
   {
      const float2 d = p_sub(fr, fl), e = __ffma2_rn(__fadd2_rn(fl, fr), f2(-0.5f), v0);
      const float2 de = __fmul2_rn(d, e), dd = __fmul2_rn(__fmul2_rn(d, d), sixth);
      const float2 alt = __ffma2_rn(fl, f2(-2.0f), v3);
      if (-dd.x > de.x) fr.x = alt.x;
      if (-dd.y > de.y) fr.y = alt.y;
   }
   a0 = fl;
   a1 = p_sub(__ffma2_rn(fl, f2(-2.0f), v3), fr);
   a2 = __ffma2_rn(v0, f2(-2.0f), __fadd2_rn(fl, fr));
}

// The same PPM in the walk form (that of the acceleration's
// remap_walk_kernel), for a walk along the cells: what a cell shares with its
// left neighbour comes in from it instead of being recomputed.
//  - tl: the left face's test (vm1 - fl)(fl - v0), which is the left
//    neighbour's right-face test (v0' - fr')(fr' - vp1') with the same
//    rounded factors; tr returns this cell's, for the next cell.
//  - dprev: v0 - vm1, the left neighbour's vp1 - v0; dn returns this cell's.
//  - The superbee slope in closed form, min(2 min(|a|,|b|), max(|a|,|b|)).
//  - The two Colella-Woodward corrections taken as alternatives: in exact
//    arithmetic the second cannot fire once the first has.
// Its limiter decisions are the reference's, up to rounding in the
// corrections; the fused tolerances cover it.
__device__ __forceinline__ void ppm_walk_x2(float2 v0, float2 vp1, float2 fl, float2 fr, float2 tl, float2 dprev,
                                            float2& tr, float2& dn, float2& a0, float2& a1, float2& a2) {
   dn = p_sub(vp1, v0);
   tr = __fmul2_rn(p_sub(v0, fr), p_sub(fr, vp1));
   float2 hs;
   {
      const float anx = fabsf(dn.x), apx = fabsf(dprev.x), any = fabsf(dn.y), apy = fabsf(dprev.y);
      hs.x = copysignf(0.5f * fminf(2.0f * fminf(anx, apx), fmaxf(anx, apx)), dn.x);
      hs.y = copysignf(0.5f * fminf(2.0f * fminf(any, apy), fmaxf(any, apy)), dn.y);
   }
   const float2 nl = p_sub(v0, hs), nr = __fadd2_rn(v0, hs);
   const bool sx = dn.x * dprev.x > 0.0f, sy = dn.y * dprev.y > 0.0f;
   float2 l, r;
   l.x = sx ? (tl.x < 0.0f ? nl.x : fl.x) : v0.x;
   l.y = sy ? (tl.y < 0.0f ? nl.y : fl.y) : v0.y;
   r.x = sx ? (tr.x < 0.0f ? nr.x : fr.x) : v0.x;
   r.y = sy ? (tr.y < 0.0f ? nr.y : fr.y) : v0.y;
   const float2 d = p_sub(r, l), e = __ffma2_rn(__fadd2_rn(l, r), f2(-0.5f), v0);
   const float2 de = __fmul2_rn(d, e), dd = __fmul2_rn(d, __fmul2_rn(d, f2((float)(1.0 / 6.0))));
   const float2 v3 = __fmul2_rn(v0, f2(3.0f));
   const float2 alt_l = __ffma2_rn(r, f2(-2.0f), v3), alt_r = __ffma2_rn(l, f2(-2.0f), v3);
   a0.x = (de.x > dd.x) ? alt_l.x : l.x;
   a0.y = (de.y > dd.y) ? alt_l.y : l.y;
   float2 nfr;
   nfr.x = (-dd.x > de.x) ? alt_r.x : r.x;
   nfr.y = (-dd.y > de.y) ? alt_r.y : r.y;
   a1 = p_sub(__ffma2_rn(a0, f2(-2.0f), v3), nfr);
   a2 = __ffma2_rn(v0, f2(-2.0f), __fadd2_rn(a0, nfr));
}

// Integral of two PPM reconstructions from 0 to u (u * (a0 + u (a1 + u a2))).
__device__ __forceinline__ float2 ppm_integral_x2(float2 u, float2 a0, float2 a1, float2 a2) {
   return __fmul2_rn(u, __ffma2_rn(u, __ffma2_rn(u, a2, a1), a0));
}

}  // namespace vlgpu
