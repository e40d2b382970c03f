// FP64 gyration transform and SLICE-3D intersections for one spatial cell,
// usable on the host and on the device.
//
// The transform follows compute_acceleration_transformation
// (vlasovsolver/cpu_acc_transform.cpp:66-153): N = |dt| / (T_g * 0.1 deg/360)
// substeps (at least one), each translating by -pivot, rotating by
// -2*pi*dt/T_g/N about the unit magnetic field, and translating back, with
// pivot = (transform so far) * V_bulk - Hall term.  The intersections follow
// compute_cell_intersections and compute_intersections_{1st,2nd,3rd}
// (vlasovsolver/cpu_acc_intersections.cpp:44-450).  An affine map is stored as
// a row-major 3x3 linear part and a translation.
#pragma once
#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define VLGPU_HD __host__ __device__
#else
#define VLGPU_HD
#endif

namespace vlgpu {
namespace geom {

struct Affine {
   double L[9];
   double t[3];
};

VLGPU_HD inline void mat_vec(const double L[9], const double v[3], double out[3]) {
   for (int r = 0; r < 3; ++r) out[r] = L[3 * r + 0] * v[0] + L[3 * r + 1] * v[1] + L[3 * r + 2] * v[2];
}
VLGPU_HD inline void apply(const Affine& a, const double v[3], double out[3]) {
   double lv[3];
   mat_vec(a.L, v, lv);
   for (int r = 0; r < 3; ++r) out[r] = lv[r] + a.t[r];
}
VLGPU_HD inline void pre_translate(Affine& a, const double v[3]) {
   for (int r = 0; r < 3; ++r) a.t[r] = a.t[r] + v[r];
}
VLGPU_HD inline void pre_rotate(Affine& a, double angle, const double u[3]) {
   const double s = sin(angle), c = cos(angle), omc = 1.0 - c;
   double R[9];
   R[0] = c + omc * u[0] * u[0];
   R[1] = omc * u[0] * u[1] - s * u[2];
   R[2] = omc * u[0] * u[2] + s * u[1];
   R[3] = omc * u[1] * u[0] + s * u[2];
   R[4] = c + omc * u[1] * u[1];
   R[5] = omc * u[1] * u[2] - s * u[0];
   R[6] = omc * u[2] * u[0] - s * u[1];
   R[7] = omc * u[2] * u[1] + s * u[0];
   R[8] = c + omc * u[2] * u[2];
   Affine out;
   for (int r = 0; r < 3; ++r)
      for (int col = 0; col < 3; ++col)
         out.L[3 * r + col] = R[3 * r + 0] * a.L[0 + col] + R[3 * r + 1] * a.L[3 + col] + R[3 * r + 2] * a.L[6 + col];
   mat_vec(R, a.t, out.t);
   a = out;
}
VLGPU_HD inline void inverse(const Affine& a, Affine& inv) {
   const double* m = a.L;
   const double c00 = m[4] * m[8] - m[5] * m[7];
   const double c01 = m[5] * m[6] - m[3] * m[8];
   const double c02 = m[3] * m[7] - m[4] * m[6];
   const double det = m[0] * c00 + m[1] * c01 + m[2] * c02;
   const double id = 1.0 / det;
   inv.L[0] = c00 * id;
   inv.L[1] = (m[2] * m[7] - m[1] * m[8]) * id;
   inv.L[2] = (m[1] * m[5] - m[2] * m[4]) * id;
   inv.L[3] = c01 * id;
   inv.L[4] = (m[0] * m[8] - m[2] * m[6]) * id;
   inv.L[5] = (m[2] * m[3] - m[0] * m[5]) * id;
   inv.L[6] = c02 * id;
   inv.L[7] = (m[1] * m[6] - m[0] * m[7]) * id;
   inv.L[8] = (m[0] * m[4] - m[1] * m[3]) * id;
   double lt[3];
   mat_vec(inv.L, a.t, lt);
   for (int r = 0; r < 3; ++r) inv.t[r] = -lt[r];
}

struct TransformInputs {
   double B[3];
   double curl[3];
   double rhoq;
   double V[3];
   double egradpe[3];
   double q, m, dt;
   double hall_min_rhoq;
   int ohm_gradpe;
   double mu0;
};

VLGPU_HD inline Affine acceleration_transform(const TransformInputs& in) {
   const double bnorm = sqrt(in.B[0] * in.B[0] + in.B[1] * in.B[1] + in.B[2] * in.B[2]);
   double unit_B[3] = {in.B[0] / bnorm, in.B[1] / bnorm, in.B[2] / bnorm};
   const double B_mag = bnorm + 1e-30;
   if (B_mag < 1e-28) {
      unit_B[0] = 0;
      unit_B[1] = 0;
      unit_B[2] = 1;
   }
   const double gyro_period = 2 * M_PI * in.m / (in.q * B_mag);
   const double EPSILON = 1e10 * 2.2250738585072014e-308;  // 1e10 * DBL_MIN
   const double rhoq = in.rhoq + EPSILON;
   const double hallRhoq = (rhoq <= in.hall_min_rhoq) ? in.hall_min_rhoq : rhoq;
   const double hallPrefactor = 1.0 / (in.mu0 * hallRhoq);
   Affine T;
   for (int q = 0; q < 9; ++q) T.L[q] = (q % 4 == 0) ? 1.0 : 0.0;
   T.t[0] = T.t[1] = T.t[2] = 0.0;
   unsigned int nsub = (unsigned int)(fabs(in.dt) / fabs(gyro_period * (0.1 / 360.0)));
   if (nsub < 1) nsub = 1;
   const double sub_rad = -(2.0 * M_PI * in.dt / gyro_period) / nsub;
   const double sub_dt = in.dt / nsub;
   for (unsigned int i = 0; i < nsub; ++i) {
      double pivot[3];
      apply(T, in.V, pivot);
      pivot[0] -= hallPrefactor * in.curl[0];
      pivot[1] -= hallPrefactor * in.curl[1];
      pivot[2] -= hallPrefactor * in.curl[2];
      const double mp[3] = {-pivot[0], -pivot[1], -pivot[2]};
      pre_translate(T, mp);
      pre_rotate(T, sub_rad, unit_B);
      pre_translate(T, pivot);
      if (in.ohm_gradpe > 0) {
         const double f = fabs(in.q) / in.m;
         const double g[3] = {f * in.egradpe[0] * sub_dt, f * in.egradpe[1] * sub_dt, f * in.egradpe[2] * sub_dt};
         pre_translate(T, g);
      }
   }
   return T;
}

VLGPU_HD inline double dot3(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
VLGPU_HD inline void line_plane(const double lp[3], const double ld[3], const double pp[3], const double pn[3],
                                double out[3]) {
   const double d[3] = {pp[0] - lp[0], pp[1] - lp[1], pp[2] - lp[2]};
   const double f = dot3(pn, d) / dot3(pn, ld);
   for (int r = 0; r < 3; ++r) out[r] = lp[r] + f * ld[r];
}
VLGPU_HD inline void add3(const double a[3], const double b[3], double out[3]) {
   for (int r = 0; r < 3; ++r) out[r] = a[r] + b[r];
}
VLGPU_HD inline void copy3(const double a[3], double out[3]) {
   for (int r = 0; r < 3; ++r) out[r] = a[r];
}
// Component i (0..2, known only at run time) of a 3-vector, read with
// selects so that no local array is indexed dynamically on the device.
VLGPU_HD inline double comp(const double v[3], int i) { return i == 0 ? v[0] : (i == 1 ? v[1] : v[2]); }
VLGPU_HD inline void store4(const double p000[3], const double p100[3], const double p010[3], const double p001[3],
                            int d, double out[4]) {
   out[0] = comp(p000, d);
   out[1] = comp(p100, d) - comp(p000, d);
   out[2] = comp(p010, d) - comp(p000, d);
   out[3] = comp(p001, d) - comp(p000, d);
}

VLGPU_HD inline void unit(int i, double scale, double out[3]) {
   for (int r = 0; r < 3; ++r) out[r] = (r == i) ? scale : 0.0;
}

// first intersections: Euclidian lines along d meet Lagrangian planes
VLGPU_HD inline void isect_1st(const Affine& bwd, const double mn[3], const double dv[3], int d, double out[4]) {
   double e[3], pn[3], pp[3], q[3], lp[3];
   unit(d, 1.0, e);
   mat_vec(bwd.L, e, pn);
   unit(d, comp(mn, d), q);
   apply(bwd, q, pp);
   for (int r = 0; r < 3; ++r) lp[r] = (r == d) ? 0.0 : 0.5 * dv[r] + mn[r];
   double p000[3], p[3][3];
   line_plane(lp, e, pp, pn, p000);
   for (int a = 0; a < 3; ++a) {
      double s[3], step[3], t[3];
      unit(a, comp(dv, a), s);
      if (a == d) {
         mat_vec(bwd.L, s, step);
         add3(pp, step, t);
         line_plane(lp, e, t, pn, p[a]);
      } else {
         add3(lp, s, t);
         line_plane(t, e, pp, pn, p[a]);
      }
   }
   store4(p000, p[0], p[1], p[2], d, out);
}

// second intersections: Lagrangian lines along n = (d+1)%3 meet Euclidian
// planes normal to n
VLGPU_HD inline void isect_2nd(const Affine& bwd, const double mn[3], const double dv[3], int d, double out[4]) {
   const int n = (d + 1) % 3;
   double pn[3], pp[3], en[3], ld[3], q[3], lp[3];
   unit(n, 1.0, pn);
   unit(n, comp(mn, n) + comp(dv, n) * 0.5, pp);
   unit(n, 1.0, en);
   mat_vec(bwd.L, en, ld);
   for (int r = 0; r < 3; ++r) q[r] = (r == d) ? mn[r] : 0.5 * dv[r] + mn[r];
   apply(bwd, q, lp);
   double p000[3], p[3][3];
   line_plane(lp, ld, pp, pn, p000);
   for (int a = 0; a < 3; ++a) {
      double s[3], step[3], t[3];
      unit(a, comp(dv, a), s);
      if (a == n) {
         add3(pp, s, t);
         line_plane(lp, ld, t, pn, p[a]);
      } else {
         mat_vec(bwd.L, s, step);
         add3(lp, step, t);
         line_plane(t, ld, pp, pn, p[a]);
      }
   }
   store4(p000, p[0], p[1], p[2], d, out);
}

// third intersections: images of cell-centre points
VLGPU_HD inline void isect_3rd(const Affine& bwd, const double mn[3], const double dv[3], int d, double out[4]) {
   double base[3];
   for (int r = 0; r < 3; ++r) base[r] = (r == d) ? 0.0 : 0.5;
   double p000[3], p[3][3], q[3];
   for (int r = 0; r < 3; ++r) q[r] = base[r] * dv[r] + mn[r];
   apply(bwd, q, p000);
   for (int a = 0; a < 3; ++a) {
      for (int r = 0; r < 3; ++r) q[r] = (base[r] + (r == a ? 1.0 : 0.0)) * dv[r] + mn[r];
      apply(bwd, q, p[a]);
   }
   store4(p000, p[0], p[1], p[2], d, out);
}

// 12 doubles ordered x(4), y(4), z(4), each (intersection, di, dj, dk).
// On the device every run-time component index goes through selects (comp,
// unit): indexing a local array initialised from kernel parameters with a
// run-time index produced wrong values with this toolchain.
VLGPU_HD inline void cell_intersections(const Affine& fwd, const double mn[3], const double dv[3], uint32_t map_order,
                                        double out12[12]) {
   Affine bwd;
   inverse(fwd, bwd);
   const int o0 = (int)(map_order % 3);
   const int o1 = (o0 + 1) % 3, o2 = (o0 + 2) % 3;
   isect_1st(bwd, mn, dv, o0, out12 + 4 * o0);
   isect_2nd(bwd, mn, dv, o1, out12 + 4 * o1);
   isect_3rd(bwd, mn, dv, o2, out12 + 4 * o2);
}

}  // namespace geom
}  // namespace vlgpu
