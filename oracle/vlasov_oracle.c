/*
 * vlasov_oracle.c -- CPU restatement of Vlasiator's Vlasov hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path is
 * compared against; the product never links, loads or calls it.  It is built
 * twice by oracle/Makefile:
 *   liborc_sp.so : realf = float  (the reference's -DSPF build, VECL = 16)
 *   liborc_dp.so : realf = double (the reference's -DDPF build, VECL = 8)
 *
 * Parity pin: for every function that has a counterpart in the reference's
 * compiled sources (map_1d, the moment sums) the tests compare this
 * restatement bit for bit against the reference's own code built by
 * oracle/build_ref.sh, and against the committed fixtures in tests/golden/.
 * The gyration transform and SLICE-3D intersections depend on Eigen, which
 * the reference tree does not ship; they are restated here in FP64 and
 * pinned against closed-form rotations (tests/test_oracle_geometry.py).
 *
 * Floating point: compiled with -ffp-contract=off so that every operation is
 * rounded exactly as the reference's scalar fallback vector class
 * (vlasovsolver/vectorclass_fallback.h) rounds it.  Where the reference mixes
 * a double constant into a realf expression (1.0/12.0 in the h4 face value,
 * i_dv = 1.0/dv in the mapping integral) the product is formed in double and
 * rounded once to realf, exactly as VecSimple<float> operator* does.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#ifndef ORC_DOUBLE
typedef float realf;
#define ORC_LANES 16
#else
typedef double realf;
#define ORC_LANES 8
#endif

#define WID 4
#define WID2 16
#define WID3 64
#define MAXDIM 256

#define ORC_OK 0
#define ORC_EINVAL 1
#define ORC_ENOMEM 2
#define ORC_EWALL 3

typedef struct {
   double vmin[3];
   double vmax[3];
   uint32_t len[3]; /* blocks per dimension */
} orc_mesh;

static double mesh_dv(const orc_mesh* m, int d) { return (m->vmax[d] - m->vmin[d]) / m->len[d] / WID; }

int orc_realf_size(void) { return (int)sizeof(realf); }

/* ------------------------------------------------------------------------- */
/* PPM reconstruction, vlasovsolver/cpu_1d_ppm.hpp:35-54 with h4 faces       */
/* (cpu_face_estimates.hpp:160-167), the superbee limiter                    */
/* (cpu_slope_limiters.hpp:30-54, 97-118) and the face filter                */
/* (cpu_face_estimates.hpp:278-323).  v points at the cell, v[-2..2] valid.  */
/* ------------------------------------------------------------------------- */
static realf h4_left_face(const realf* v) {
   /* 1/12 * (-v[-2] + 7 v[-1] + 7 v[0] - v[1]); each product rounded to realf,
      sums left to right, the 1/12 product in double then rounded. */
   realf s = (realf)(-1.0 * v[-2]);
   s = s + (realf)(7.0 * v[-1]);
   s = s + (realf)(7.0 * v[0]);
   s = s - (realf)(1.0 * v[1]);
   return (realf)((1.0 / 12.0) * (double)s);
}

static realf minmod(realf s1, realf s2) {
   const realf slope = (fabs(s1) < fabs(s2)) ? s1 : s2;
   return (s1 * s2 <= 0) ? (realf)0 : slope;
}
static realf maxmod(realf s1, realf s2) {
   const realf slope = (fabs(s1) > fabs(s2)) ? s1 : s2;
   return (s1 * s2 <= 0) ? (realf)0 : slope;
}
static realf superbee(realf l, realf m, realf r) {
   const realf a = r - m;
   const realf b = m - l;
   const realf s1 = minmod(a, (realf)2 * b);
   const realf s2 = minmod((realf)2 * a, b);
   return maxmod(s1, s2);
}

static void ppm_coeff(const realf* v, realf threshold, realf a[3]) {
   realf fl = h4_left_face(v);
   realf fr = h4_left_face(v + 1);
   const realf scale = (realf)(1.0 / (double)threshold);
   const realf slope = superbee(v[-1] * scale, v[0] * scale, v[1] * scale);
   realf slope_abs = (realf)fabs(slope);
   const realf slope_sign = (slope > 0) ? (realf)1 : (realf)-1;
   slope_abs = slope_abs * threshold;
   if (slope_abs == (realf)0) {
      fr = v[0];
      fl = v[0];
   }
   if ((v[-1] - fl) * (fl - v[0]) < 0) fl = v[0] - (realf)(slope_sign * 0.5) * slope_abs;
   if ((v[1] - fr) * (fr - v[0]) < 0) fr = v[0] + (realf)(slope_sign * 0.5) * slope_abs;
   /* Colella-Woodward monotonicity, cpu_1d_ppm.hpp:41-47 */
   const realf one_sixth = (realf)(1.0 / 6.0);
   {
      const realf d = fr - fl;
      const realf e = v[0] - (realf)(0.5 * (fl + fr));
      if (d * e > d * d * one_sixth) fl = (realf)3 * v[0] - (realf)2 * fr;
   }
   {
      const realf d = fr - fl;
      const realf e = v[0] - (realf)(0.5 * (fl + fr));
      if (-d * d * one_sixth > d * e) fr = (realf)3 * v[0] - (realf)2 * fl;
   }
   a[0] = fl;
   a[1] = (realf)(3.0 * v[0]) - (realf)(2.0 * fl) - fr;
   a[2] = fl + fr - (realf)(2.0 * v[0]);
}

/* ------------------------------------------------------------------------- */
/* One SLICE-3D 1D remap of one cell, vlasovsolver/cpu_acc_map.cpp:121-636.  */
/* Input blocks in any order; output blocks sorted by global ID.             */
/* ------------------------------------------------------------------------- */

/* (i,j,k) of a block in the frame where the sweep dimension is k
   (cpu_acc_map.cpp:85-106). */
static void swapped_indices(uint32_t gid, const orc_mesh* m, int dim, uint32_t out[3]) {
   const uint32_t x = gid % m->len[0];
   const uint32_t y = (gid / m->len[0]) % m->len[1];
   const uint32_t z = gid / (m->len[0] * m->len[1]);
   if (dim == 0) { out[0] = z; out[1] = y; out[2] = x; }
   else if (dim == 1) { out[0] = x; out[1] = z; out[2] = y; }
   else { out[0] = x; out[1] = y; out[2] = z; }
}
static uint32_t gid_from_swapped(const uint32_t s[3], const orc_mesh* m, int dim) {
   uint32_t x, y, z;
   if (dim == 0) { z = s[0]; y = s[1]; x = s[2]; }
   else if (dim == 1) { x = s[0]; z = s[1]; y = s[2]; }
   else { x = s[0]; y = s[1]; z = s[2]; }
   return x + m->len[0] * (y + m->len[1] * z);
}
/* position of cell (lane i, lane j, sweep offset g) inside a block,
   cell_indices_to_id of cpu_acc_map.cpp:151-199 */
static int cell_offset(int dim, int i, int j, int g) {
   if (dim == 0) return i * WID2 + j * WID + g;
   if (dim == 1) return i + j * WID2 + g * WID;
   return i + j * WID + g * WID2;
}

typedef struct {
   uint32_t key;   /* transverse set index * len_k + k */
   uint32_t index; /* input block index */
} keyidx;

static int cmp_keyidx(const void* a, const void* b) {
   const uint32_t x = ((const keyidx*)a)->key, y = ((const keyidx*)b)->key;
   return (x > y) - (x < y);
}
static int cmp_u32(const void* a, const void* b) {
   const uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
   return (x > y) - (x < y);
}

static realf max_f(realf a, realf b) { return (a < b) ? b : a; } /* std::max */
static realf min_f(realf a, realf b) { return (b < a) ? b : a; } /* std::min */

/* Target block range of one column, cpu_acc_map.cpp:258-324.  Returns 1 if
   the range comes closer than wall_margin blocks to the mesh wall
   (the bail-out condition of cpu_acc_map.cpp:325-338). */
static int column_extent(realf intersection, realf di, realf dj, realf dk, realf dv, realf v_min, int max_v_length,
                         uint32_t set_i, uint32_t set_j, uint32_t first_k, uint32_t last_k, int wall_margin,
                         int* first_out, int* last_out) {
   const realf c00 = intersection + (realf)(set_i * WID + 0) * di + (realf)(set_j * WID + 0) * dj;
   const realf c01 = intersection + (realf)(set_i * WID + 0) * di + (realf)(set_j * WID + WID - 1) * dj;
   const realf c10 = intersection + (realf)(set_i * WID + WID - 1) * di + (realf)(set_j * WID + 0) * dj;
   const realf c11 = intersection + (realf)(set_i * WID + WID - 1) * di + (realf)(set_j * WID + WID - 1) * dj;
   realf mx = c00, mn = c00;
   mx = max_f(mx, c01); mx = max_f(mx, c10); mx = max_f(mx, c11);
   mn = min_f(mn, c01); mn = min_f(mn, c10); mn = min_f(mn, c11);
   const realf first_min_v = (realf)(WID * first_k) * dv + v_min;
   const realf last_max_v = (realf)(WID * (last_k + 1)) * dv + v_min;
   const int first_gk = (int)((first_min_v - mx) / dk);
   const int last_gk = (int)((last_max_v - mn) / dk);
   int fb = first_gk / WID, lb = last_gk / WID;
   fb = (fb >= 0) ? fb : 0;
   fb = (fb < max_v_length) ? fb : max_v_length - 1;
   lb = (lb >= 0) ? lb : 0;
   lb = (lb < max_v_length) ? lb : max_v_length - 1;
   *first_out = fb;
   *last_out = lb;
   return (fb < wall_margin || fb >= max_v_length - wall_margin || lb < wall_margin || lb >= max_v_length - wall_margin);
}

/* status bits returned through *flags */
#define ORC_FLAG_WALL 1u

int orc_map_1d(const orc_mesh* m, uint32_t n_in, const uint32_t* gids_in, const realf* data_in,
               double in_intersection, double in_di, double in_dj, double in_dk, uint32_t dim, double min_value,
               uint32_t wall_margin, uint32_t cap, uint32_t* n_out, uint32_t* gids_out, realf* data_out,
               uint32_t* flags) {
   *flags = 0;
   *n_out = 0;
   if (dim > 2) return ORC_EINVAL;
   if (n_in == 0) return ORC_OK;
   realf intersection = (realf)in_intersection;
   realf di = (realf)in_di, dj = (realf)in_dj, dk = (realf)in_dk;
   if (dim == 0) { realf t = di; di = dk; dk = t; }
   if (dim == 1) { realf t = dj; dj = dk; dk = t; }
   const realf dv = (realf)mesh_dv(m, dim);
   const realf v_min = (realf)m->vmin[dim];
   const int max_v_length = (int)m->len[dim];
   const double i_dv = 1.0 / (double)dv;
   const realf threshold = (realf)min_value;
   uint32_t len_i, len_j;
   {
      const uint32_t L[3] = {m->len[0], m->len[1], m->len[2]};
      if (dim == 0) { len_i = L[2]; len_j = L[1]; }
      else if (dim == 1) { len_i = L[0]; len_j = L[2]; }
      else { len_i = L[0]; len_j = L[1]; }
      (void)len_i;
   }

   /* sort by (set, k): cpu_acc_sort_blocks.cpp:46-155 */
   keyidx* order = (keyidx*)malloc(sizeof(keyidx) * n_in);
   if (!order) return ORC_ENOMEM;
   for (uint32_t b = 0; b < n_in; ++b) {
      uint32_t s[3];
      swapped_indices(gids_in[b], m, (int)dim, s);
      order[b].key = (s[0] * len_j + s[1]) * (uint32_t)max_v_length + s[2];
      order[b].index = b;
   }
   qsort(order, n_in, sizeof(keyidx), cmp_keyidx);

   /* scratch: padded column values [lane][cell] for one set, one target
      accumulator per set */
   const int ncell_max = (MAXDIM + 2) * WID;
   realf* values = (realf*)calloc((size_t)WID2 * ncell_max, sizeof(realf));
   realf* target = (realf*)calloc((size_t)MAXDIM * WID3, sizeof(realf));
   int* col_first = (int*)malloc(sizeof(int) * MAXDIM);
   int* col_last = (int*)malloc(sizeof(int) * MAXDIM);
   uint32_t* col_start = (uint32_t*)malloc(sizeof(uint32_t) * MAXDIM);
   uint32_t* col_len = (uint32_t*)malloc(sizeof(uint32_t) * MAXDIM);
   if (!values || !target || !col_first || !col_last || !col_start || !col_len) {
      free(order); free(values); free(target); free(col_first); free(col_last); free(col_start); free(col_len);
      return ORC_ENOMEM;
   }
   int status = ORC_OK;
   uint32_t nout = 0;

   uint32_t s0 = 0;
   while (s0 < n_in) {
      /* one column set: all blocks with the same transverse (i,j) */
      const uint32_t set_key = order[s0].key / (uint32_t)max_v_length;
      uint32_t s1 = s0;
      while (s1 < n_in && order[s1].key / (uint32_t)max_v_length == set_key) ++s1;
      uint32_t set_idx[3];
      swapped_indices(gids_in[order[s0].index], m, (int)dim, set_idx);
      /* split into columns (contiguous runs of k) */
      int ncol = 0;
      for (uint32_t b = s0; b < s1; ++b) {
         const uint32_t k = order[b].key % (uint32_t)max_v_length;
         if (b == s0 || k != (order[b - 1].key % (uint32_t)max_v_length) + 1) {
            col_start[ncol] = b;
            col_len[ncol] = 0;
            ++ncol;
         }
         col_len[ncol - 1]++;
      }
      unsigned char is_target[MAXDIM], is_source[MAXDIM];
      memset(is_target, 0, sizeof(is_target));
      memset(is_source, 0, sizeof(is_source));
      for (int c = 0; c < ncol; ++c) {
         const uint32_t fk = order[col_start[c]].key % (uint32_t)max_v_length;
         const uint32_t lk = fk + col_len[c] - 1;
         if (column_extent(intersection, di, dj, dk, dv, v_min, max_v_length, set_idx[0], set_idx[1], fk, lk,
                           (int)wall_margin, &col_first[c], &col_last[c]))
            *flags |= ORC_FLAG_WALL;
         for (uint32_t k = fk; k <= lk; ++k) is_source[k] = 1;
         for (int k = col_first[c]; k <= col_last[c]; ++k) is_target[k] = 1;
      }
      memset(target, 0, sizeof(realf) * (size_t)max_v_length * WID3);

      /* map each column, cpu_acc_map.cpp:393-631 */
      for (int c = 0; c < ncol; ++c) {
         const uint32_t n_cblocks = col_len[c];
         const uint32_t kbegin = order[col_start[c]].key % (uint32_t)max_v_length;
         const int ncell = (int)(n_cblocks + 2) * WID;
         /* load transposed with one zero block at each end (cpu_acc_load_blocks.cpp) */
         for (int lane = 0; lane < WID2; ++lane) {
            realf* col = values + (size_t)lane * ncell_max;
            for (int q = 0; q < ncell; ++q) col[q] = 0;
            const int li = lane % WID, lj = lane / WID;
            for (uint32_t b = 0; b < n_cblocks; ++b) {
               const realf* blk = data_in + (size_t)order[col_start[c] + b].index * WID3;
               for (int g = 0; g < WID; ++g) col[(b + 1) * WID + g] = blk[cell_offset((int)dim, li, lj, g)];
            }
         }
         for (int jg = 0; jg < WID2 / ORC_LANES; ++jg) {
            /* one vector of ORC_LANES lanes: lane l -> i = l % WID, j = jg*(ORC_LANES/WID) + l / WID */
            realf im[ORC_LANES], v_r[ORC_LANES];
            int gk_r[ORC_LANES];
            for (int l = 0; l < ORC_LANES; ++l) {
               const int i = l % WID, j = jg * (ORC_LANES / WID) + l / WID;
               const realf A = (realf)(set_idx[0] * WID) + (realf)i;
               const realf B = (realf)(set_idx[1] * WID) + (realf)j;
               im[l] = intersection + A * di;
               im[l] = im[l] + B * dj;
               v_r[l] = (realf)(WID * kbegin) * dv + v_min;
            }
            int min_lane = 0, max_lane = 0;
            {
               double maxV = DBL_MIN, minV = DBL_MAX;
               for (int l = 0; l < ORC_LANES; ++l) {
                  const realf lag = (v_r[l] - im[l]) / dk;
                  gk_r[l] = (int)lag;
                  if ((double)lag > maxV) { maxV = lag; max_lane = l; }
                  if ((double)lag < minV) { minV = lag; min_lane = l; }
               }
            }
            for (uint32_t k = 0; k < WID * n_cblocks; ++k) {
               realf a[ORC_LANES][3];
               realf v_l[ORC_LANES];
               int gk_l[ORC_LANES];
               for (int l = 0; l < ORC_LANES; ++l) {
                  const int lane = jg * ORC_LANES + l;
                  const realf* col = values + (size_t)lane * ncell_max;
                  ppm_coeff(col + k + WID, threshold, a[l]);
                  v_l[l] = v_r[l];
                  v_r[l] = v_r[l] + dv;
                  gk_l[l] = gk_r[l];
                  gk_r[l] = (int)((v_r[l] - im[l]) / dk);
               }
               int minGk = gk_l[min_lane];
               if (minGk < col_first[c] * WID) minGk = col_first[c] * WID;
               int maxGk = gk_r[max_lane];
               if (maxGk > (col_last[c] + 1) * WID - 1) maxGk = (col_last[c] + 1) * WID - 1;
               realf dens_r[ORC_LANES];
               for (int l = 0; l < ORC_LANES; ++l) dens_r[l] = 0;
               for (int gk = minGk; gk <= maxGk; ++gk) {
                  const int blockK = gk / WID;
                  const int gmod = gk - blockK * WID;
                  for (int l = 0; l < ORC_LANES; ++l) {
                     const int i = l % WID, j = jg * (ORC_LANES / WID) + l / WID;
                     realf x = (realf)(gk + 1) * dk + im[l];
                     x = (x > v_l[l]) ? x : v_l[l]; /* max(x, v_l) */
                     x = (x < v_r[l]) ? x : v_r[l]; /* min(x, v_r) */
                     const realf u = (realf)((double)(x - v_l[l]) * i_dv);
                     const realf dl = dens_r[l];
                     dens_r[l] = u * (a[l][0] + u * (a[l][1] + u * a[l][2]));
                     realf* t = target + (size_t)blockK * WID3 + cell_offset((int)dim, i, j, gmod);
                     *t = *t + (dens_r[l] - dl);
                  }
               }
            }
         }
      }
      /* emit this set's target blocks */
      for (int k = 0; k < max_v_length; ++k) {
         if (!is_target[k]) continue;
         if (nout >= cap) { status = ORC_ENOMEM; continue; }
         const uint32_t s[3] = {set_idx[0], set_idx[1], (uint32_t)k};
         gids_out[nout] = gid_from_swapped(s, m, (int)dim);
         memcpy(data_out + (size_t)nout * WID3, target + (size_t)k * WID3, sizeof(realf) * WID3);
         ++nout;
      }
      s0 = s1;
   }
   free(order); free(values); free(target); free(col_first); free(col_last); free(col_start); free(col_len);
   if (status != ORC_OK) return status;
   /* canonical order: ascending global ID */
   {
      keyidx* o2 = (keyidx*)malloc(sizeof(keyidx) * (nout ? nout : 1));
      realf* tmp = (realf*)malloc(sizeof(realf) * WID3 * (size_t)(nout ? nout : 1));
      if (!o2 || !tmp) { free(o2); free(tmp); return ORC_ENOMEM; }
      for (uint32_t b = 0; b < nout; ++b) { o2[b].key = gids_out[b]; o2[b].index = b; }
      qsort(o2, nout, sizeof(keyidx), cmp_keyidx);
      memcpy(tmp, data_out, sizeof(realf) * WID3 * (size_t)nout);
      for (uint32_t b = 0; b < nout; ++b) {
         gids_out[b] = o2[b].key;
         memcpy(data_out + (size_t)b * WID3, tmp + (size_t)o2[b].index * WID3, sizeof(realf) * WID3);
      }
      free(o2); free(tmp);
   }
   *n_out = nout;
   return ORC_OK;
}

/* ------------------------------------------------------------------------- */
/* FP64 gyration transform and SLICE-3D intersections.                       */
/* Restates vlasovsolver/cpu_acc_transform.cpp:66-153 and                    */
/* vlasovsolver/cpu_acc_intersections.cpp:44-450 without Eigen: an affine    */
/* map is a 3x3 linear part L (row major) and a translation t.               */
/* ------------------------------------------------------------------------- */
typedef struct { double L[9]; double t[3]; } orc_affine;

static void aff_identity(orc_affine* a) {
   memset(a, 0, sizeof(*a));
   a->L[0] = a->L[4] = a->L[8] = 1.0;
}
static void mat_vec(const double L[9], const double v[3], double out[3]) {
   for (int r = 0; r < 3; ++r) out[r] = L[3 * r + 0] * v[0] + L[3 * r + 1] * v[1] + L[3 * r + 2] * v[2];
}
static void aff_apply(const orc_affine* a, const double v[3], double out[3]) {
   double lv[3];
   mat_vec(a->L, v, lv);
   for (int r = 0; r < 3; ++r) out[r] = lv[r] + a->t[r];
}
/* a <- translation(v) * a */
static void aff_pre_translate(orc_affine* a, const double v[3]) {
   for (int r = 0; r < 3; ++r) a->t[r] = a->t[r] + v[r];
}
/* a <- R * a for the rotation by angle about the unit axis u (Rodrigues) */
static void aff_pre_rotate(orc_affine* a, double angle, const double u[3]) {
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
   orc_affine out;
   for (int r = 0; r < 3; ++r) {
      for (int col = 0; col < 3; ++col)
         out.L[3 * r + col] = R[3 * r + 0] * a->L[0 + col] + R[3 * r + 1] * a->L[3 + col] + R[3 * r + 2] * a->L[6 + col];
   }
   mat_vec(R, a->t, out.t);
   *a = out;
}
static void aff_inverse(const orc_affine* a, orc_affine* inv) {
   const double* m = a->L;
   const double c00 = m[4] * m[8] - m[5] * m[7];
   const double c01 = m[5] * m[6] - m[3] * m[8];
   const double c02 = m[3] * m[7] - m[4] * m[6];
   const double det = m[0] * c00 + m[1] * c01 + m[2] * c02;
   const double id = 1.0 / det;
   inv->L[0] = c00 * id;
   inv->L[1] = (m[2] * m[7] - m[1] * m[8]) * id;
   inv->L[2] = (m[1] * m[5] - m[2] * m[4]) * id;
   inv->L[3] = c01 * id;
   inv->L[4] = (m[0] * m[8] - m[2] * m[6]) * id;
   inv->L[5] = (m[2] * m[3] - m[0] * m[5]) * id;
   inv->L[6] = c02 * id;
   inv->L[7] = (m[1] * m[6] - m[0] * m[7]) * id;
   inv->L[8] = (m[0] * m[4] - m[1] * m[3]) * id;
   double lt[3];
   mat_vec(inv->L, a->t, lt);
   for (int r = 0; r < 3; ++r) inv->t[r] = -lt[r];
}

/* Inputs per cell, as read from SpatialCell::parameters by the reference:
   B[3] = BGB*VOL + PERB*VOL, curl_terms[3] = (dBZdy - dBYdz, dBXdz - dBZdx,
   dBYdx - dBXdy) of the perturbed field, rhoq = RHOQ_V, V[3] = VX_V..VZ_V,
   egradpe[3] = E*GRADPE; species charge q and mass m. */
void orc_acceleration_transform(const double B[3], const double curl_terms[3], double rhoq_v, const double V[3],
                                const double egradpe[3], double q, double m, double dt, double hall_min_rhoq,
                                int ohm_gradpe, double mu0, double out_L[9], double out_t[3]) {
   const double bnorm = sqrt(B[0] * B[0] + B[1] * B[1] + B[2] * B[2]);
   double unit_B[3] = {B[0] / bnorm, B[1] / bnorm, B[2] / bnorm};
   const double B_mag = bnorm + 1e-30;
   if (B_mag < 1e-28) { unit_B[0] = 0; unit_B[1] = 0; unit_B[2] = 1; }
   const double gyro_period = 2 * M_PI * m / (q * B_mag);
   const double EPSILON = 1e10 * DBL_MIN;
   const double rhoq = rhoq_v + EPSILON;
   const double hallRhoq = (rhoq <= hall_min_rhoq) ? hall_min_rhoq : rhoq;
   const double hallPrefactor = 1.0 / (mu0 * hallRhoq);
   orc_affine T;
   aff_identity(&T);
   unsigned int nsub = (unsigned int)(fabs(dt) / fabs(gyro_period * (0.1 / 360.0)));
   if (nsub < 1) nsub = 1;
   const double sub_rad = -(2.0 * M_PI * dt / gyro_period) / nsub;
   const double sub_dt = dt / nsub;
   for (unsigned int i = 0; i < nsub; ++i) {
      double pivot[3];
      aff_apply(&T, V, pivot);
      pivot[0] -= hallPrefactor * curl_terms[0];
      pivot[1] -= hallPrefactor * curl_terms[1];
      pivot[2] -= hallPrefactor * curl_terms[2];
      const double mp[3] = {-pivot[0], -pivot[1], -pivot[2]};
      aff_pre_translate(&T, mp);
      aff_pre_rotate(&T, sub_rad, unit_B);
      aff_pre_translate(&T, pivot);
      if (ohm_gradpe > 0) {
         const double f = fabs(q) / m;
         const double g[3] = {f * egradpe[0] * sub_dt, f * egradpe[1] * sub_dt, f * egradpe[2] * sub_dt};
         aff_pre_translate(&T, g);
      }
   }
   memcpy(out_L, T.L, sizeof(T.L));
   memcpy(out_t, T.t, sizeof(T.t));
}

static double dot3(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
/* cpu_acc_intersections.cpp:112-118 */
static void line_plane(const double lp[3], const double ld[3], const double pp[3], const double pn[3], double out[3]) {
   const double d[3] = {pp[0] - lp[0], pp[1] - lp[1], pp[2] - lp[2]};
   const double nom = dot3(pn, d);
   const double dem = dot3(pn, ld);
   const double f = nom / dem;
   for (int r = 0; r < 3; ++r) out[r] = lp[r] + f * ld[r];
}
static void add3(const double a[3], const double b[3], double out[3]) {
   for (int r = 0; r < 3; ++r) out[r] = a[r] + b[r];
}
static void store4(const double p000[3], const double p100[3], const double p010[3], const double p001[3], int d,
                   double out[4]) {
   out[0] = p000[d];
   out[1] = p100[d] - p000[d];
   out[2] = p010[d] - p000[d];
   out[3] = p001[d] - p000[d];
}

/* first intersection set, cpu_acc_intersections.cpp:132-231 */
static void isect_1st(const orc_affine* bwd, const double mn[3], const double dv[3], int d, double out[4]) {
   double e[3] = {0, 0, 0};
   e[d] = 1.0;
   double pn[3], pp[3], q[3] = {0, 0, 0};
   mat_vec(bwd->L, e, pn);
   q[d] = mn[d];
   aff_apply(bwd, q, pp);
   double lp[3];
   for (int r = 0; r < 3; ++r) lp[r] = (r == d) ? 0.0 : 0.5 * dv[r] + mn[r];
   double step[3][3];
   for (int a = 0; a < 3; ++a) {
      double s[3] = {0, 0, 0};
      s[a] = dv[a];
      if (a == d) mat_vec(bwd->L, s, step[a]);
      else memcpy(step[a], s, sizeof(s));
   }
   double p000[3], p[3][3];
   line_plane(lp, e, pp, pn, p000);
   for (int a = 0; a < 3; ++a) {
      double t[3];
      if (a == d) { add3(pp, step[a], t); line_plane(lp, e, t, pn, p[a]); }
      else { add3(lp, step[a], t); line_plane(t, e, pp, pn, p[a]); }
   }
   store4(p000, p[0], p[1], p[2], d, out);
}

/* second intersection set, cpu_acc_intersections.cpp:246-358: the
   Lagrangian line along the rotated next dimension n = (d+1)%3 meets the
   Euclidian planes normal to that same dimension. */
static void isect_2nd(const orc_affine* bwd, const double mn[3], const double dv[3], int d, double out[4]) {
   const int n = (d + 1) % 3; /* line direction (before rotation) */
   const int o = n;           /* Euclidian plane normal */
   double pn[3] = {0, 0, 0}, pp[3] = {0, 0, 0};
   pn[o] = 1.0;
   pp[o] = mn[o] + dv[o] * 0.5;
   double en[3] = {0, 0, 0}, ld[3];
   en[n] = 1.0;
   mat_vec(bwd->L, en, ld);
   double q[3];
   for (int r = 0; r < 3; ++r) q[r] = (r == d) ? mn[r] : 0.5 * dv[r] + mn[r];
   double lp[3];
   aff_apply(bwd, q, lp);
   double step[3][3];
   for (int a = 0; a < 3; ++a) {
      double s[3] = {0, 0, 0};
      s[a] = dv[a];
      if (a == o) memcpy(step[a], s, sizeof(s));
      else mat_vec(bwd->L, s, step[a]);
   }
   double p000[3], p[3][3];
   line_plane(lp, ld, pp, pn, p000);
   for (int a = 0; a < 3; ++a) {
      double t[3];
      if (a == o) { add3(pp, step[a], t); line_plane(lp, ld, t, pn, p[a]); }
      else { add3(lp, step[a], t); line_plane(t, ld, pp, pn, p[a]); }
   }
   store4(p000, p[0], p[1], p[2], d, out);
}

/* third intersection set, cpu_acc_intersections.cpp:376-450: images of
   cell-centre points (the sweep coordinate at the cell face) */
static void isect_3rd(const orc_affine* bwd, const double mn[3], const double dv[3], int d, double out[4]) {
   double base[3];
   for (int r = 0; r < 3; ++r) base[r] = (r == d) ? 0.0 : 0.5;
   double p000[3], p[3][3];
   {
      double q[3];
      for (int r = 0; r < 3; ++r) q[r] = base[r] * dv[r] + mn[r];
      aff_apply(bwd, q, p000);
   }
   for (int a = 0; a < 3; ++a) {
      double q[3];
      for (int r = 0; r < 3; ++r) q[r] = (base[r] + (r == a ? 1.0 : 0.0)) * dv[r] + mn[r];
      aff_apply(bwd, q, p[a]);
   }
   store4(p000, p[0], p[1], p[2], d, out);
}

/* compute_cell_intersections (cpu_acc_intersections.cpp:44-101): given the
   forward transform, writes 12 doubles ordered x(4), y(4), z(4), each
   (intersection, di, dj, dk). */
void orc_cell_intersections(const double fwd_L[9], const double fwd_t[3], const orc_mesh* m, uint32_t map_order,
                            double out12[12]) {
   orc_affine fwd, bwd;
   memcpy(fwd.L, fwd_L, sizeof(fwd.L));
   memcpy(fwd.t, fwd_t, sizeof(fwd.t));
   aff_inverse(&fwd, &bwd);
   const double mn[3] = {m->vmin[0], m->vmin[1], m->vmin[2]};
   const double dv[3] = {mesh_dv(m, 0), mesh_dv(m, 1), mesh_dv(m, 2)};
   static const int orders[3][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}};
   const int* o = orders[map_order % 3];
   isect_1st(&bwd, mn, dv, o[0], out12 + 4 * o[0]);
   isect_2nd(&bwd, mn, dv, o[1], out12 + 4 * o[1]);
   isect_3rd(&bwd, mn, dv, o[2], out12 + 4 * o[2]);
}

/* ------------------------------------------------------------------------- */
/* Velocity moments of one cell, vlasovsolver/arch_moments.h:83-155 and the   */
/* per-population bookkeeping of calculateMoments_V                           */
/* (vlasovsolver/arch_moments.cpp:342-499).  out16: n, n*V(3), RHOM_V, V(3),  */
/* RHOQ_V, P_11, P_22, P_33, P_23, P_13, P_12, sum f.  Plain sums in double,  */
/* blocks in the given order, cells i fastest.                                */
/* ------------------------------------------------------------------------- */
void orc_moments(const orc_mesh* m, uint32_t n, const uint32_t* gids, const realf* data, double mass, double charge,
                 int second, double out16[16]) {
   const double bs[3] = {(m->vmax[0] - m->vmin[0]) / m->len[0], (m->vmax[1] - m->vmin[1]) / m->len[1],
                         (m->vmax[2] - m->vmin[2]) / m->len[2]};
   const double dv[3] = {bs[0] / WID, bs[1] / WID, bs[2] / WID};
   const double DV3 = dv[0] * dv[1] * dv[2];
   double a[5] = {0, 0, 0, 0, 0};
   for (uint32_t b = 0; b < n; ++b) {
      const uint32_t g = gids[b];
      const uint32_t bi = g % m->len[0], bj = (g / m->len[0]) % m->len[1], bk = g / (m->len[0] * m->len[1]);
      for (int c = 0; c < WID3; ++c) {
         const int i = c % WID, j = (c / WID) % WID, k = c / WID2;
         const double VX = (m->vmin[0] + bi * bs[0]) + (i + 0.5) * dv[0];
         const double VY = (m->vmin[1] + bj * bs[1]) + (j + 0.5) * dv[1];
         const double VZ = (m->vmin[2] + bk * bs[2]) + (k + 0.5) * dv[2];
         const double f = (double)data[(size_t)b * WID3 + c];
         a[0] += f * DV3;
         a[1] += f * VX * DV3;
         a[2] += f * VY * DV3;
         a[3] += f * VZ * DV3;
         a[4] += f;
      }
   }
   for (int q = 0; q < 16; ++q) out16[q] = 0.0;
   out16[0] = a[0]; out16[1] = a[1]; out16[2] = a[2]; out16[3] = a[3];
   const double rhom = a[0] * mass;
   out16[4] = rhom;
   out16[5] = rhom != 0.0 ? (a[1] * mass) / rhom : 0.0;
   out16[6] = rhom != 0.0 ? (a[2] * mass) / rhom : 0.0;
   out16[7] = rhom != 0.0 ? (a[3] * mass) / rhom : 0.0;
   out16[8] = a[0] * charge;
   out16[15] = a[4];
   if (!second) return;
   const double V[3] = {out16[5], out16[6], out16[7]};
   double p[6] = {0, 0, 0, 0, 0, 0};
   for (uint32_t b = 0; b < n; ++b) {
      const uint32_t g = gids[b];
      const uint32_t bi = g % m->len[0], bj = (g / m->len[0]) % m->len[1], bk = g / (m->len[0] * m->len[1]);
      for (int c = 0; c < WID3; ++c) {
         const int i = c % WID, j = (c / WID) % WID, k = c / WID2;
         const double VX = (m->vmin[0] + bi * bs[0]) + (i + 0.5) * dv[0];
         const double VY = (m->vmin[1] + bj * bs[1]) + (j + 0.5) * dv[1];
         const double VZ = (m->vmin[2] + bk * bs[2]) + (k + 0.5) * dv[2];
         const double f = (double)data[(size_t)b * WID3 + c];
         p[0] += f * (VX - V[0]) * (VX - V[0]) * DV3;
         p[1] += f * (VY - V[1]) * (VY - V[1]) * DV3;
         p[2] += f * (VZ - V[2]) * (VZ - V[2]) * DV3;
         p[3] += f * (VY - V[1]) * (VZ - V[2]) * DV3;
         p[4] += f * (VX - V[0]) * (VZ - V[2]) * DV3;
         p[5] += f * (VX - V[0]) * (VY - V[1]) * DV3;
      }
   }
   for (int q = 0; q < 6; ++q) out16[9 + q] = mass * p[q];
}

/* ------------------------------------------------------------------------- */
/* Block adjustment of one cell without spatial neighbours,                  */
/* SpatialCell::adjust_velocity_blocks (spatial_cells/spatial_cell_cpu.cpp:  */
/* 179-273) with the content test of compute_block_has_content (:290-320):   */
/* the new set is the content blocks and their +-add_width neighbours inside */
/* the mesh; kept blocks keep their data, added ones are zero, the removed   */
/* mass sum(f)*dv^3 is returned in *loss.  Output sorted by global ID.        */
/* ------------------------------------------------------------------------- */
/* With spatial neighbours: extra[0..n_extra) are the global IDs of the      */
/* blocks with content in the cell's spatial neighbours                       */
/* (spatial_cell_cpu.cpp:211-221); they join the kept set as they are.       */
int orc_adjust_with(const orc_mesh* m, uint32_t n, const uint32_t* gids, const realf* data, double min_value,
                    int add_width, uint32_t n_extra, const uint32_t* extra, uint32_t cap, uint32_t* n_out,
                    uint32_t* gids_out, realf* data_out, double* loss) {
   const uint32_t L0 = m->len[0], L1 = m->len[1], L2 = m->len[2];
   const size_t nb = (size_t)L0 * L1 * L2;
   int32_t* where = (int32_t*)malloc(sizeof(int32_t) * nb);
   unsigned char* keep = (unsigned char*)calloc(nb, 1);
   if (!where || !keep) { free(where); free(keep); return ORC_ENOMEM; }
   for (size_t q = 0; q < nb; ++q) where[q] = -1;
   for (uint32_t q = 0; q < n_extra; ++q)
      if (extra[q] < nb) keep[extra[q]] = 1;
   for (uint32_t b = 0; b < n; ++b) where[gids[b]] = (int32_t)b;
   for (uint32_t b = 0; b < n; ++b) {
      int content = 0;
      for (int c = 0; c < WID3; ++c)
         if ((double)data[(size_t)b * WID3 + c] >= min_value) { content = 1; break; }
      if (!content) continue;
      const int x = (int)(gids[b] % L0), y = (int)((gids[b] / L0) % L1), z = (int)(gids[b] / (L0 * L1));
      for (int dx = -add_width; dx <= add_width; ++dx)
         for (int dy = -add_width; dy <= add_width; ++dy)
            for (int dz = -add_width; dz <= add_width; ++dz) {
               const int X = x + dx, Y = y + dy, Z = z + dz;
               if (X < 0 || Y < 0 || Z < 0 || X >= (int)L0 || Y >= (int)L1 || Z >= (int)L2) continue;
               keep[(size_t)X + L0 * ((size_t)Y + L1 * (size_t)Z)] = 1;
            }
   }
   const double dvx = (m->vmax[0] - m->vmin[0]) / L0 / WID, dvy = (m->vmax[1] - m->vmin[1]) / L1 / WID,
                dvz = (m->vmax[2] - m->vmin[2]) / L2 / WID;
   const double DV3 = dvx * dvy * dvz;
   double lost = 0.0;
   for (uint32_t b = 0; b < n; ++b) {
      if (keep[gids[b]]) continue;
      double sum = 0.0;
      for (int c = 0; c < WID3; ++c) sum += data[(size_t)b * WID3 + c];
      lost += DV3 * sum;
   }
   uint32_t o = 0;
   int status = ORC_OK;
   for (size_t g = 0; g < nb; ++g) {
      if (!keep[g]) continue;
      if (o >= cap) { status = ORC_ENOMEM; break; }
      gids_out[o] = (uint32_t)g;
      if (where[g] >= 0) memcpy(data_out + (size_t)o * WID3, data + (size_t)where[g] * WID3, sizeof(realf) * WID3);
      else memset(data_out + (size_t)o * WID3, 0, sizeof(realf) * WID3);
      ++o;
   }
   *n_out = o;
   *loss = lost;
   free(where);
   free(keep);
   return status;
}

int orc_adjust(const orc_mesh* m, uint32_t n, const uint32_t* gids, const realf* data, double min_value,
               int add_width, uint32_t cap, uint32_t* n_out, uint32_t* gids_out, realf* data_out, double* loss) {
   return orc_adjust_with(m, n, gids, data, min_value, add_width, 0, NULL, cap, n_out, gids_out, data_out, loss);
}

/* The global IDs of the blocks with content (compute_block_has_content,      */
/* spatial_cell_cpu.cpp:290-320); returns their number.                       */
uint32_t orc_content_gids(uint32_t n, const uint32_t* gids, const realf* data, double min_value, uint32_t* out) {
   uint32_t k = 0;
   for (uint32_t b = 0; b < n; ++b) {
      for (int c = 0; c < WID3; ++c)
         if ((double)data[(size_t)b * WID3 + c] >= min_value) {
            out[k++] = gids[b];
            break;
         }
   }
   return k;
}

/* ------------------------------------------------------------------------- */
/* Spatial translation on a uniform, periodic grid: one dimension of         */
/* trans_map_1d_amr (vlasovsolver/cpu_trans_map_amr.cpp:214-443) with        */
/* propagatePencil (:37-150) and compute_ppm_coeff_nonuniform                 */
/* (cpu_1d_ppm_nonuniform.hpp:40-62, faces cpu_face_estimates.hpp:179-191,    */
/* 327-378).  Every cell has width dz along the dimension and target ratio 1. */
/* Cells are x fastest; cell c owns blocks offsets[c]..offsets[c+1]-1 (any    */
/* order).  Block sets do not change; mass entering a cell that lacks the     */
/* block is dropped, as in the reference.  data_out has the layout of data.   */
/* ------------------------------------------------------------------------- */
static realf h4_face_nonuniform(const realf* h, const realf* u) {
   /* h[-2..1], u[-2..1]: left face of cell 0 (White et al. 2008 eq. 45) */
   const double D1 = 1.0 / (h[-2] + h[-1] + h[0] + h[1]);
   const realf F1 = (h[-2] + h[-1]) * (h[0] + h[1]) / (h[-1] + h[0]);
   const realf V1 = F1 * (u[-1] * h[0] + u[0] * h[-1]);
   const double D2 = 1.0 / (h[-2] + h[-1] + h[0]) + 1.0 / (h[-1] + h[0] + h[1]);
   const realf V2 = (realf)((double)V1 * D2);
   const realf F2 = (h[0] * (h[0] + h[1])) / ((h[-2] + h[-1] + h[0]) * (h[-2] + h[-1]));
   const double D3 = h[-2] + 2.0 * h[-1];
   const realf V3a = (realf)((double)u[-1] * D3) - (u[-2] * h[-1]);
   const realf V3 = F2 * V3a;
   const realf F3 = h[-1] * (h[-2] + h[-1]) / ((h[-1] + h[0] + h[1]) * (h[0] + h[1]));
   const double D4 = 2.0 * h[0] + h[1];
   const realf V4a = (realf)((double)u[0] * D4) - u[1] * h[0];
   const realf V4 = F3 * V4a;
   const realf S = V2 + V3 + V4;
   return (realf)(D1 * (double)S);
}

static void ppm_coeff_nonuniform(const realf* h, const realf* v, realf threshold, realf a[3]) {
   realf fl = h4_face_nonuniform(h, v);
   realf fr = h4_face_nonuniform(h + 1, v + 1);
   realf slope_abs, slope_sign;
   if (threshold > 0) {
      const realf scale = (realf)(1.0 / (double)threshold);
      const realf s = superbee(v[-1] * scale, v[0] * scale, v[1] * scale);
      slope_abs = (realf)fabs(s) * threshold;
      slope_sign = (s > 0) ? (realf)1 : (realf)-1;
   } else {
      const realf s = superbee(v[-1], v[0], v[1]);
      slope_abs = (realf)fabs(s);
      slope_sign = (s > 0) ? (realf)1 : (realf)-1;
   }
   if (slope_abs == (realf)0) { fr = v[0]; fl = v[0]; }
   if ((v[-1] - fl) * (fl - v[0]) < 0) fl = v[0] - (realf)(slope_sign * 0.5) * slope_abs;
   if ((v[1] - fr) * (fr - v[0]) < 0) fr = v[0] + (realf)(slope_sign * 0.5) * slope_abs;
   const realf one_sixth = (realf)(1.0 / 6.0);
   {
      const realf d = fr - fl, e = v[0] - (realf)(0.5 * (fl + fr));
      if (d * e > d * d * one_sixth) fl = (realf)3 * v[0] - (realf)2 * fr;
   }
   {
      const realf d = fr - fl, e = v[0] - (realf)(0.5 * (fl + fr));
      if (-d * d * one_sixth > d * e) fr = (realf)3 * v[0] - (realf)2 * fl;
   }
   a[0] = fl;
   a[1] = (realf)(3.0 * v[0]) - (realf)(2.0 * fl) - fr;
   a[2] = fl + fr - (realf)(2.0 * v[0]);
}

int orc_translate(const orc_mesh* m, const uint32_t grid[3], const uint64_t* offsets, const uint32_t* gids,
                  const realf* data, uint32_t dim, realf dt, realf dz, double min_value, realf* data_out) {
   if (dim > 2) return ORC_EINVAL;
   const uint32_t nx = grid[0], ny = grid[1], nz = grid[2];
   const uint64_t ncells = (uint64_t)nx * ny * nz;
   const uint32_t N = grid[dim];
   const size_t nb = (size_t)m->len[0] * m->len[1] * m->len[2];
   const realf dvz = (realf)mesh_dv(m, (int)dim);
   const realf vz_min = (realf)m->vmin[dim];
   const realf threshold = (realf)min_value;
   /* stride between consecutive cells along dim */
   const uint64_t stride = dim == 0 ? 1 : (dim == 1 ? nx : (uint64_t)nx * ny);
   const uint32_t n_other = (uint32_t)(ncells / N);
   int32_t* where = (int32_t*)malloc(sizeof(int32_t) * nb * N);
   unsigned char* inunion = (unsigned char*)malloc(nb);
   realf* vals = (realf*)malloc(sizeof(realf) * (size_t)N * WID3);
   realf* outv = (realf*)malloc(sizeof(realf) * (size_t)N * WID3);
   realf* hbuf = (realf*)malloc(sizeof(realf) * (N + 8));
   if (!where || !inunion || !vals || !outv || !hbuf) {
      free(where); free(inunion); free(vals); free(outv); free(hbuf);
      return ORC_ENOMEM;
   }
   for (uint32_t q = 0; q < N + 8; ++q) hbuf[q] = dz;
   const realf* h = hbuf + 4; /* h[-4 .. N+3] */
   memcpy(data_out, data, sizeof(realf) * WID3 * (size_t)offsets[ncells]);
   for (uint32_t p = 0; p < n_other; ++p) {
      /* first cell of this pencil */
      uint64_t c0;
      if (dim == 0) c0 = (uint64_t)p * nx;
      else if (dim == 1) c0 = (uint64_t)(p % nx) + (uint64_t)nx * ny * (p / nx);
      else c0 = p;
      memset(inunion, 0, nb);
      for (uint32_t x = 0; x < N; ++x) {
         const uint64_t c = c0 + x * stride;
         for (size_t g = 0; g < nb; ++g) where[(size_t)x * nb + g] = -1;
         for (uint64_t b = offsets[c]; b < offsets[c + 1]; ++b) {
            where[(size_t)x * nb + gids[b]] = (int32_t)b;
            inunion[gids[b]] = 1;
         }
      }
      for (size_t g = 0; g < nb; ++g) {
         if (!inunion[g]) continue;
         for (uint32_t x = 0; x < N; ++x) {
            const int32_t b = where[(size_t)x * nb + g];
            for (int q = 0; q < WID3; ++q) vals[(size_t)x * WID3 + q] = b >= 0 ? data[(size_t)b * WID3 + q] : 0;
            memset(outv + (size_t)x * WID3, 0, sizeof(realf) * WID3);
         }
         uint32_t s[3];
         swapped_indices((uint32_t)g, m, (int)dim, s);
         for (uint32_t i = 0; i < N; ++i) {
            const uint32_t im1 = (i + N - 1) % N, ip1 = (i + 1) % N;
            for (int k = 0; k < WID; ++k) {
               const realf cell_vz = (realf)((s[2] * WID + k + 0.5) * (double)dvz + (double)vz_min);
               const realf zt = cell_vz * dt / h[i];
               const int pos = zt > 0;
               const realf z_1 = pos ? (realf)(1.0 - zt) : (realf)0;
               const realf z_2 = pos ? (realf)1 : -zt;
               /* the reference skips a whole 16-lane plane when no value in the
                  5-cell stencil is positive (check_skip_remapping) */
               int any_pos = 0;
               for (int di = -2; di <= 2 && !any_pos; ++di) {
                  const uint32_t ii = (uint32_t)(((int)i + di + 2 * (int)N) % (int)N);
                  for (int lane = 0; lane < WID2; ++lane)
                     if (vals[(size_t)ii * WID3 + cell_offset((int)dim, lane % WID, lane / WID, k)] > 0) {
                        any_pos = 1;
                        break;
                     }
               }
               if (!any_pos) continue;
               for (int lane = 0; lane < WID2; ++lane) {
                  const int off = cell_offset((int)dim, lane % WID, lane / WID, k);
                  realf st[5];
                  for (int di = -2; di <= 2; ++di) {
                     const uint32_t ii = (uint32_t)(((int)i + di + 2 * (int)N) % (int)N);
                     st[di + 2] = vals[(size_t)ii * WID3 + off];
                  }
                  realf a[3];
                  ppm_coeff_nonuniform(h + i, st + 2, threshold, a);
                  const realf ngbr = z_2 * (a[0] + z_2 * (a[1] + z_2 * a[2])) - z_1 * (a[0] + z_1 * (a[1] + z_1 * a[2]));
                  if (where[(size_t)i * nb + g] >= 0) {
                     realf* t = outv + (size_t)i * WID3 + off;
                     *t = *t + (st[2] - ngbr) * (realf)1;
                  }
                  if (where[(size_t)ip1 * nb + g] >= 0) {
                     realf* t = outv + (size_t)ip1 * WID3 + off;
                     *t = *t + (pos ? ngbr * h[i] / h[i + 1] : (realf)0) * (realf)1;
                  }
                  if (where[(size_t)im1 * nb + g] >= 0) {
                     realf* t = outv + (size_t)im1 * WID3 + off;
                     *t = *t + (!pos ? ngbr * h[i] / h[(int)i - 1] : (realf)0) * (realf)1;
                  }
               }
            }
         }
         for (uint32_t x = 0; x < N; ++x) {
            const int32_t b = where[(size_t)x * nb + g];
            if (b >= 0) memcpy(data_out + (size_t)b * WID3, outv + (size_t)x * WID3, sizeof(realf) * WID3);
         }
      }
   }
   free(where); free(inunion); free(vals); free(outv); free(hbuf);
   return ORC_OK;
}
