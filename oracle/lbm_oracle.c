/* CPU oracle for the iLBMReX per-level hot path: TEST INFRASTRUCTURE ONLY.
 *
 * Plain C, FP64, one level held in one box.  It restates the reference's
 * algorithm function by function (citations are path:line in the reference
 * project) and keeps the reference's operation order so that, compiled with
 * -ffp-contract=off, it reproduces the reference's own code bit for bit
 * (checked against oracle/_ref, which compiles the reference sources in place).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this library, and only as the checker / baseline.  The product path never
 * calls it.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "oracle_case.h"

#define BC_INT_DIR 0
#define BC_FOEXTRAP 2
#define BC_EXT_DIR 3
#define BC_USER_1 1001
#define BC_USER_2 1002

typedef struct {
  int n;               /* markers */
  double *x, *y, *z;   /* current positions */
  double *u, *v, *w;   /* interpolated velocity */
  double *fx, *fy, *fz;
  double *mx, *my, *mz; /* user target velocity, then moment r x F */
  double *phi, *theta;  /* circle/sphere parametrisation (1-based, index 0 unused) */
  double *xref, *yref, *zref;
  double dv, wall_tol;
  ilbm_ib_case p;
  int kernel;
  /* IVC cache */
  int ivc_ready, ivc_n;
  double *lu;
  int *piv;
  double *xc, *yc, *zc;
  double fsum[3];
  /* pitching-airfoil parameters (IBMUserDefinedGeometry.H:14-20) */
  double chord, thick, pitch_mean, pitch_amp, pitch_freq, pitch_phase, pivot_x;
} orc_ib;

typedef struct orc_level_s {
  ilbm_case c;
  int dim, Q, ng, ngz;
  int n[3], gn[3];
  long gcells;
  double w[ILBM_MAX_Q], cx[ILBM_MAX_Q], cy[ILBM_MAX_Q], cz[ILBM_MAX_Q];
  double dx[3], plo[3], phi[3];
  int bclo[3], bchi[3];
  double lo_rho[3], lo_ux[3], lo_uy[3], lo_uz[3];
  double hi_rho[3], hi_ux[3], hi_uy[3], hi_uz[3];
  int periodic[3];
  double tau, dt, time;
  long step;
  double *f_new, *f_old, *mac_new, *mac_old, *forcing; /* grown boxes, component-major */
  double *last_fx;                                     /* grown box, 3 comps */
  int use_ib;
  orc_ib ib;
  double rec[ILBM_FORCE_REC];
  int have_prev;
  double prev[3];
  /* fine level of a two-level hierarchy: its coarse level, the fine-domain
   * index of its cell 0, and the time weights of the coarse macro fields
   * for the substep being taken (mode 0 old, 1 new, 2 a*old + b*new) */
  struct orc_level_s *cf;
  int cflo[3];
  int cf_mode;
  double cf_a, cf_b;
} orc_level;

/* ------------------------------------------------------------------------ */
/* indexing over the grown box (Array4 layout, components outermost)        */
/* ------------------------------------------------------------------------ */
static inline long IX(const orc_level *L, int i, int j, int k) {
  return (long)(i + L->ng) + (long)(j + L->ng) * L->gn[0] +
         (long)(k + L->ngz) * L->gn[0] * L->gn[1];
}
static inline int in_domain(const orc_level *L, int i, int j, int k) {
  if (i < 0 || i >= L->n[0] || j < 0 || j >= L->n[1]) return 0;
  if (L->dim == 3 && (k < 0 || k >= L->n[2])) return 0;
  return 1;
}
static inline int in_grown(const orc_level *L, int i, int j, int k) {
  if (i < -L->ng || i >= L->n[0] + L->ng || j < -L->ng || j >= L->n[1] + L->ng) return 0;
  if (L->dim == 3 && (k < -L->ng || k >= L->n[2] + L->ng)) return 0;
  if (L->dim == 2 && k != 0) return 0;
  return 1;
}
static inline double dmax(double a, double b) { return (a < b) ? b : a; }
static inline double dmin(double a, double b) { return (b < a) ? b : a; }
static inline int imax(int a, int b) { return (a < b) ? b : a; }
static inline int imin(int a, int b) { return (b < a) ? b : a; }

/* feqFunction, Source/LBM/feq.H:9-29 */
static double orc_feq(const orc_level *L, double wi, double cx, double cy, double cz,
                      double rho, double u, double v, double w) {
  double eu, uv;
  if (L->dim == 3) {
    eu = cx * u + cy * v + cz * w;
    uv = u * u + v * v + w * w;
  } else {
    eu = cx * u + cy * v;
    uv = u * u + v * v;
  }
  return wi * rho * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * uv);
}

/* collide + collide_forced, Source/LBM/collide.H:9-25, collide_forced.H:10-51
 * (in place on f[q], q-stride fs) */
static void orc_collide_forced(const orc_level *L, double *f, long fs, const double *feq,
                               double tau, double ux, double uy, double uz, double fx,
                               double fy, double fz) {
  const int Q = L->Q;
  for (int q = 0; q < Q; ++q) f[q * fs] = 1.0 * f[q * fs] - (f[q * fs] - feq[q]) / tau;
  if (fx == 0.0 && fy == 0.0 && fz == 0.0) return;
  const double cs2 = 1.0 / 3.0;
  const double fac = 1.0 - 0.5 / tau;
  for (int q = 0; q < Q; ++q) {
    double cx = L->cx[q], cy = L->cy[q], cz = L->cz[q];
    double eiu = cx * ux + cy * uy + cz * uz;
    double termx = (cx - ux) / cs2 + (eiu / (cs2 * cs2)) * cx;
    double termy = (cy - uy) / cs2 + (eiu / (cs2 * cs2)) * cy;
    double termz = (L->dim == 3) ? ((cz - uz) / cs2 + (eiu / (cs2 * cs2)) * cz) : 0.0;
    double Si = L->w[q] * fac * (termx * fx + termy * fy + termz * fz);
    f[q * fs] += Si;
  }
}

/* ------------------------------------------------------------------------ */
/* ghost fill (FillPatchSingleLevel + PhysBCFunct semantics)                */
/* ------------------------------------------------------------------------ */

/* nearestInteriorCellAndBoundaryHits + firstBoundaryFaceOfType,
 * Source/BC/bc_fill.H:12-67 */
static int first_face_of_type(const orc_level *L, const int *iv, int type, int *bc_dim,
                              int *lo_side) {
  for (int d = 0; d < L->dim; ++d) {
    const int lo = 0, hi = L->n[d] - 1;
    if (iv[d] < lo && L->bclo[d] == type) { *bc_dim = d; *lo_side = 1; return 1; }
    if (iv[d] > hi && L->bchi[d] == type) { *bc_dim = d; *lo_side = 0; return 1; }
  }
  return 0;
}
static void mirror_of(const orc_level *L, const int *iv, int *m) {
  for (int d = 0; d < 3; ++d) m[d] = iv[d];
  for (int d = 0; d < L->dim; ++d) {
    if (iv[d] < 0) m[d] = 0;
    else if (iv[d] > L->n[d] - 1) m[d] = L->n[d] - 1;
  }
}
static void bc_vals(const orc_level *L, int d, int lo, double *rb, double *ub, double *vb,
                    double *wb) {
  *rb = lo ? L->lo_rho[d] : L->hi_rho[d];
  *ub = lo ? L->lo_ux[d] : L->hi_ux[d];
  *vb = lo ? L->lo_uy[d] : L->hi_uy[d];
  *wb = lo ? L->lo_uz[d] : L->hi_uz[d];
}

/* applyExtDirMesoscopic / applyFaceMirroredMesoscopic, bc_fill.H:156-261 */
static void neq_fill(const orc_level *L, double *f, long gi, long mi, int bc_dim, int lo,
                     int face_mirror) {
  const int Q = L->Q;
  const long fs = L->gcells;
  double fnp[ILBM_MAX_Q];
  double rhonp = 0.0, unp = 0.0, vnp = 0.0, wnp = 0.0;
  for (int n = 0; n < Q; ++n) {
    fnp[n] = f[mi + n * fs];
    rhonp += fnp[n];
    unp += L->cx[n] * fnp[n];
    vnp += L->cy[n] * fnp[n];
    wnp += L->cz[n] * fnp[n];
  }
  rhonp = dmax(rhonp, 1.0e-20);
  unp /= rhonp;
  vnp /= rhonp;
  wnp /= rhonp;
  double rb, ub, vb, wb;
  bc_vals(L, bc_dim, lo, &rb, &ub, &vb, &wb);
  double rt = rb, ut = ub, vt = vb, wt = wb;
  if (face_mirror) {
    rt = dmax(1.0e-20, 2.0 * rb - rhonp);
    ut = 2.0 * ub - unp;
    vt = 2.0 * vb - vnp;
    wt = 2.0 * wb - wnp;
  }
  for (int n = 0; n < Q; ++n) {
    double eu_np = L->cx[n] * unp + L->cy[n] * vnp + L->cz[n] * wnp;
    double uv_np = unp * unp + vnp * vnp + wnp * wnp;
    double feqnp = L->w[n] * rhonp * (1.0 + 3.0 * eu_np + 4.5 * eu_np * eu_np - 1.5 * uv_np);
    double eu_t = L->cx[n] * ut + L->cy[n] * vt + L->cz[n] * wt;
    double uv_t = ut * ut + vt * vt + wt * wt;
    double feqt = L->w[n] * rt * (1.0 + 3.0 * eu_t + 4.5 * eu_t * eu_t - 1.5 * uv_t);
    f[gi + n * fs] = feqt + (fnp[n] - feqnp);
  }
}

/* mesoscopicBcFill::operator(), bc_fill.H:303-347 */
static void meso_user(const orc_level *L, double *f, const int *iv) {
  int m[3], bd, lo;
  mirror_of(L, iv, m);
  const long gi = IX(L, iv[0], iv[1], iv[2]);
  const long mi = IX(L, m[0], m[1], m[2]);
  if (first_face_of_type(L, iv, BC_USER_2, &bd, &lo)) {
    neq_fill(L, f, gi, mi, bd, lo, 1);
    return;
  }
  if (first_face_of_type(L, iv, BC_USER_1, &bd, &lo)) {
    for (int n = 0; n < L->Q; ++n) f[gi + n * L->gcells] = f[mi + n * L->gcells];
    return;
  }
  if (first_face_of_type(L, iv, BC_EXT_DIR, &bd, &lo)) {
    neq_fill(L, f, gi, mi, bd, lo, 0);
    return;
  }
}

/* macroBcFill::operator(), bc_fill.H:69-142, 263-301 */
static void macro_user(const orc_level *L, double *m6, int nc, const int *iv) {
  int m[3], bd, lo;
  mirror_of(L, iv, m);
  const long gi = IX(L, iv[0], iv[1], iv[2]);
  const long mi = IX(L, m[0], m[1], m[2]);
  const long s = L->gcells;
  double rb, ub, vb, wb;
  if (first_face_of_type(L, iv, BC_USER_2, &bd, &lo)) {
    for (int n = 0; n < nc; ++n) m6[gi + n * s] = m6[mi + n * s];
    bc_vals(L, bd, lo, &rb, &ub, &vb, &wb);
    if (nc > 0) m6[gi] = dmax(1.0e-20, 2.0 * rb - m6[mi]);
    if (nc > 1) m6[gi + s] = 2.0 * ub - m6[mi + s];
    if (nc > 2) m6[gi + 2 * s] = 2.0 * vb - m6[mi + 2 * s];
    if (nc > 3) m6[gi + 3 * s] = 2.0 * wb - m6[mi + 3 * s];
    return;
  }
  if (first_face_of_type(L, iv, BC_USER_1, &bd, &lo) ||
      first_face_of_type(L, iv, BC_EXT_DIR, &bd, &lo)) {
    for (int n = 0; n < nc; ++n) m6[gi + n * s] = m6[mi + n * s];
    bc_vals(L, bd, lo, &rb, &ub, &vb, &wb);
    if (nc > 0) m6[gi] = rb;
    if (nc > 1) m6[gi + s] = ub;
    if (nc > 2) m6[gi + 2 * s] = vb;
    if (nc > 3) m6[gi + 3 * s] = wb;
    return;
  }
}

/* AMReX built-in first-order extrapolation (foextrap) of one ghost cell */
static void filcc(const orc_level *L, double *a, int nc, const int *iv) {
  const long gi = IX(L, iv[0], iv[1], iv[2]);
  for (int n = 0; n < nc; ++n) {
    for (int d = 0; d < L->dim; ++d) {
      int src[3] = {iv[0], iv[1], iv[2]};
      int code;
      if (iv[d] < 0) { code = L->bclo[d]; src[d] = 0; }
      else if (iv[d] > L->n[d] - 1) { code = L->bchi[d]; src[d] = L->n[d] - 1; }
      else continue;
      if (code == BC_FOEXTRAP) a[gi + n * L->gcells] = a[IX(L, src[0], src[1], src[2]) + n * L->gcells];
    }
  }
}

/* periodic image of a cell, or -1 when it lies outside in a non-periodic dim */
static int wrap_cell(const orc_level *L, const int *iv, int *w) {
  for (int d = 0; d < 3; ++d) w[d] = iv[d];
  for (int d = 0; d < L->dim; ++d) {
    if (iv[d] >= 0 && iv[d] < L->n[d]) continue;
    if (!L->periodic[d]) return -1;
    w[d] = ((iv[d] % L->n[d]) + L->n[d]) % L->n[d];
  }
  return 0;
}

/* FillBoundary(periodicity): ghost cells with a periodic image in the domain */
static void fill_boundary(const orc_level *L, double *a, int nc) {
  const int kz0 = (L->dim == 3) ? -L->ng : 0, kz1 = (L->dim == 3) ? L->n[2] + L->ng : 1;
  for (int k = kz0; k < kz1; ++k)
    for (int j = -L->ng; j < L->n[1] + L->ng; ++j)
      for (int i = -L->ng; i < L->n[0] + L->ng; ++i) {
        if (in_domain(L, i, j, k)) continue;
        int iv[3] = {i, j, k}, w[3];
        if (wrap_cell(L, iv, w) != 0) continue;
        const long gi = IX(L, i, j, k), wi = IX(L, w[0], w[1], w[2]);
        for (int n = 0; n < nc; ++n) a[gi + n * L->gcells] = a[wi + n * L->gcells];
      }
}

/* ---- coarse-fine ghosts of a fine level (static two-level hierarchy) ---- */

/* coarse macro component n at coarse cell (i,j,k) at the substep's time:
 * GetDataMacro's choice of old / new / both (AmrCoreLBM.cpp:2239-2269) and,
 * for both, FillPatchSingleLevel's linear time interpolation (AMReX
 * MultiFab::LinComb, a*old + b*new) */
static double cf_coarse(const orc_level *F, int n, int i, int j, int k) {
  const orc_level *C = F->cf;
  /* (i,j,k) in the coarse level's domain index space; C's own box starts at
   * C->cflo there (0 for the coarsest level) */
  const long e = IX(C, i - C->cflo[0], j - C->cflo[1], (C->dim == 3) ? k - C->cflo[2] : 0) +
                 (long)n * C->gcells;
  if (F->cf_mode == 0) return C->mac_old[e];
  if (F->cf_mode == 1) return C->mac_new[e];
  return F->cf_a * C->mac_old[e] + F->cf_b * C->mac_new[e];
}

/* monotonised-central limited slope of AMReX's cell-conservative linear
 * interpolation (cell_cons_interp), from the coarse cell and its two
 * neighbours in one direction */
static double mc_slope(double cl, double c, double cr) {
  const double dc = 0.5 * (cr - cl), dl = c - cl, dr = cr - c;
  if (dl * dr <= 0.0) return 0.0;
  double m = fabs(dc);
  m = dmin(m, 2.0 * fabs(dl));
  m = dmin(m, 2.0 * fabs(dr));
  return (dc < 0.0) ? -m : m;
}

static int floor_half(int v) { return (v >= 0) ? v / 2 : -((1 - v) / 2); }

/* FillPatchTwoLevels of the macro fields into fine cell (i,j,k) (fine-level
 * local index) from the coarse level, ratio 2: the coarse cell under it, its
 * limited slopes, and the fine cell centre's offset of -1/4 or +1/4 coarse
 * cell per direction (AmrCoreLBM::FillPatchMacro, AmrCoreLBM.cpp:2166-2198) */
static void cf_macro(const orc_level *F, int i, int j, int k, double *m, int nc) {
  const int fi[3] = {i + F->cflo[0], j + F->cflo[1], (F->dim == 3) ? k + F->cflo[2] : 0};
  int ic[3] = {0, 0, 0};
  double off[3] = {0.0, 0.0, 0.0};
  for (int d = 0; d < F->dim; ++d) {
    ic[d] = floor_half(fi[d]);
    off[d] = (fi[d] - 2 * ic[d] == 0) ? -0.25 : 0.25;
  }
  for (int n = 0; n < nc; ++n) {
    const double c = cf_coarse(F, n, ic[0], ic[1], ic[2]);
    double v = c;
    for (int d = 0; d < F->dim; ++d) {
      int lo[3] = {ic[0], ic[1], ic[2]}, hi[3] = {ic[0], ic[1], ic[2]};
      lo[d] -= 1;
      hi[d] += 1;
      const double cl = cf_coarse(F, n, lo[0], lo[1], lo[2]);
      const double cr = cf_coarse(F, n, hi[0], hi[1], hi[2]);
      v = v + mc_slope(cl, c, cr) * off[d];
    }
    m[n] = v;
  }
}

/* the equilibrium FillPatchMesoscopic writes into a fine level's ghosts
 * (AmrCoreLBM.cpp:1566-1626) */
static double cf_feq(double wi, double cx, double cy, double cz, double rho, double u0, double v0,
                     double w0) {
  const double r = dmax(rho, 1.e-12);
  const double u2 = u0 * u0 + v0 * v0 + w0 * w0;
  const double cu = cx * u0 + cy * v0 + cz * w0;
  return wi * r * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * u2);
}

/* a fine level's FillPatch: valid cells copied, every ghost cell (all of them
 * lie on the coarse-fine boundary: the fine box is inside the domain) from
 * the coarse macro fields -- the macro itself, or its equilibrium */
static void fill_patch_fine(const orc_level *L, double *dst, const double *src, int nc, int meso) {
  const int kz0 = (L->dim == 3) ? -L->ng : 0, kz1 = (L->dim == 3) ? L->n[2] + L->ng : 1;
  for (int k = kz0; k < kz1; ++k)
    for (int j = -L->ng; j < L->n[1] + L->ng; ++j)
      for (int i = -L->ng; i < L->n[0] + L->ng; ++i) {
        const long gi = IX(L, i, j, k);
        if (in_domain(L, i, j, k)) {
          for (int n = 0; n < nc; ++n) dst[gi + n * L->gcells] = src[gi + n * L->gcells];
          continue;
        }
        double m[6];
        cf_macro(L, i, j, k, m, 6);
        if (meso) {
          for (int q = 0; q < nc; ++q)
            dst[gi + q * L->gcells] = cf_feq(L->w[q], L->cx[q], L->cy[q], L->cz[q], m[0], m[1], m[2], m[3]);
        } else {
          for (int n = 0; n < nc; ++n) dst[gi + n * L->gcells] = m[n];
        }
      }
}

/* FillPatchSingleLevel(dst <- src) + PhysBCFunct (faces, then edges, then corners) */
static void fill_patch(const orc_level *L, double *dst, const double *src, int nc, int meso) {
  if (L->cf) {
    fill_patch_fine(L, dst, src, nc, meso);
    return;
  }
  const int kz0 = (L->dim == 3) ? -L->ng : 0, kz1 = (L->dim == 3) ? L->n[2] + L->ng : 1;
  for (int n = 0; n < nc; ++n)
    for (int k = kz0; k < kz1; ++k)
      for (int j = -L->ng; j < L->n[1] + L->ng; ++j)
        for (int i = -L->ng; i < L->n[0] + L->ng; ++i)
          if (in_domain(L, i, j, k)) {
            const long gi = IX(L, i, j, k);
            dst[gi + n * L->gcells] = src[gi + n * L->gcells];
          }
  fill_boundary(L, dst, nc);
  for (int cls = 1; cls <= L->dim; ++cls)
    for (int k = kz0; k < kz1; ++k)
      for (int j = -L->ng; j < L->n[1] + L->ng; ++j)
        for (int i = -L->ng; i < L->n[0] + L->ng; ++i) {
          int iv[3] = {i, j, k}, nout = 0;
          for (int d = 0; d < L->dim; ++d)
            if (!L->periodic[d] && (iv[d] < 0 || iv[d] > L->n[d] - 1)) ++nout;
          if (nout != cls) continue;
          filcc(L, dst, nc, iv);
          if (meso) meso_user(L, dst, iv);
          else macro_user(L, dst, nc, iv);
        }
}

/* ------------------------------------------------------------------------ */
/* marker direct-forcing IBM, Source/IBM/IBMarkerDF.cpp                     */
/* ------------------------------------------------------------------------ */

/* delta_function, IBMarkerDF.cpp:70-99 */
static double orc_delta(double xf, double xp, double h, int type) {
  const double rr = fabs(xf - xp) / h;
  double value = 0.0;
  if (type == 0) {
    if (rr < 1.0) value = 0.125 * (3.0 - 2.0 * rr + sqrt(1.0 + 4.0 * rr - 4.0 * rr * rr));
    else if (rr < 2.0) value = 0.125 * (5.0 - 2.0 * rr - sqrt(-7.0 + 12.0 * rr - 4.0 * rr * rr));
  } else {
    if (rr < 0.5) value = (1.0 + sqrt(1.0 - 3.0 * rr * rr)) / 3.0;
    else if (rr < 1.5) value = (5.0 - 3.0 * rr - sqrt(-2.0 + 6.0 * rr - 3.0 * rr * rr)) / 6.0;
  }
  return value / h;
}
/* delta_type_to_kernel, IBMarkerDF.cpp:101-113 */
static int delta_kernel(int t) {
  if (t == 4 || t == 0) return 0;
  if (t == 3 || t == 1) return 1;
  return 0;
}
/* overlap_1d, IBMarkerDF.cpp:123-145 */
static double orc_overlap_1d(double xa, double xb, double h, int kt, double plo, int ilo,
                             int ihi) {
  const int ia = (int)floor((xa - plo) / h);
  const int ib = (int)floor((xb - plo) / h);
  int lo = imax(ia - 2, ib - 2), hi = imin(ia + 2, ib + 2);
  lo = imax(lo, ilo);
  hi = imin(hi, ihi);
  if (lo > hi) return 0.0;
  double sum = 0.0;
  for (int i = lo; i <= hi; ++i) {
    const double xc = plo + ((double)i + 0.5) * h;
    const double da = orc_delta(xc, xa, h, kt);
    const double db = orc_delta(xc, xb, h, kt);
    sum += da * db * h;
  }
  return sum;
}

/* rigid_target_velocity + box_target_velocity, IBMarkerDF.cpp:147-182 */
static void rigid_target(const orc_level *L, double x, double y, double z, double *ux,
                         double *uy, double *uz) {
  const orc_ib *B = &L->ib;
  const ilbm_ib_case *p = &B->p;
  if (p->geometry_type == 1) {
    *ux = *uy = *uz = 0.0;
    if (fabs(y - p->box_yhi) <= B->wall_tol) {
      *ux = p->box_lid_ux;
      *uy = p->box_lid_uy;
      *uz = p->box_lid_uz;
    }
    return;
  }
  const double z0 = (L->dim == 3) ? p->z0 : 0.0;
  const double rx = x - p->x0, ry = y - p->y0, rz = z - z0;
  const double cx = p->omy * rz - p->omz * ry;
  const double cy = p->omz * rx - p->omx * rz;
  const double cz = p->omx * ry - p->omy * rx;
  *ux = p->ubx + cx;
  *uy = p->uby + cy;
  *uz = p->ubz + cz;
}

/* pitching NACA marker kinematics, Examples/Pitching_airfoil/IBMUserDefinedGeometry.H:144-175
 * (pivot_x shifts the pivot along the chord; 0 reproduces the leading-edge pivot) */
static void user_marker_state(const orc_level *L, int idx, double time, double *x, double *y,
                              double *z, double *ux, double *uy, double *uz) {
  const orc_ib *B = &L->ib;
  const double twopi = 2.0 * 3.14159265358979323846;
  const double phase = twopi * B->pitch_freq * time + B->pitch_phase;
  const double angle = B->pitch_mean + B->pitch_amp * sin(phase);
  const double omega = twopi * B->pitch_freq * B->pitch_amp * cos(phase);
  const double xr = B->xref[idx] - B->pivot_x, yr = B->yref[idx], zr = B->zref[idx];
  const double c = cos(angle), s = sin(angle);
  const double x0 = B->p.x0, y0 = B->p.y0, z0 = (L->dim == 3) ? B->p.z0 : 0.0;
  *x = x0 + c * xr - s * yr;
  *y = y0 + s * xr + c * yr;
  *z = z0 + zr;
  *ux = -omega * (*y - y0);
  *uy = omega * (*x - x0);
  *uz = 0.0;
}

static double *dalloc(long n) { return (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double)); }

/* build_markers, IBMarkerDF.cpp:201-497; NACA: IBMUserDefinedGeometry.H:59-142 */
static int build_markers(orc_level *L) {
  orc_ib *B = &L->ib;
  const ilbm_ib_case *p = &B->p;
  const double h = L->dx[0];
  const double pi = 3.14159265358979323846;
  int Ml = p->n_marker;
  double dv = 0.0;
  if (p->geometry_type == 1) { /* box, 2D only */
    if (L->dim != 2) return -1;
    double xlo = p->box_xlo, xhi = p->box_xhi, ylo = p->box_ylo, yhi = p->box_yhi;
    if (xhi <= xlo) { xlo = L->plo[0]; xhi = L->phi[0]; }
    if (yhi <= ylo) { ylo = L->plo[1]; yhi = L->phi[1]; }
    const double epsx = dmax(1.0e-6 * L->dx[0], 1.0e-12);
    const double epsy = dmax(1.0e-6 * L->dx[1], 1.0e-12);
    xlo = dmax(xlo, L->plo[0] + epsx);
    xhi = dmin(xhi, L->phi[0] - epsx);
    ylo = dmax(ylo, L->plo[1] + epsy);
    yhi = dmin(yhi, L->phi[1] - epsy);
    if (xhi <= xlo || yhi <= ylo) return -1;
    B->p.box_xlo = xlo; B->p.box_xhi = xhi; B->p.box_ylo = ylo; B->p.box_yhi = yhi;
    double ds = (p->box_ds > 0.0) ? p->box_ds : h;
    ds = dmax(ds, 1.0e-12);
    const int nx = imax(2, (int)lround((xhi - xlo) / ds) + 1);
    const int ny = imax(2, (int)lround((yhi - ylo) / ds) + 1);
    const double dsx = (xhi - xlo) / (double)(nx - 1);
    const double dsy = (yhi - ylo) / (double)(ny - 1);
    const int lid = (p->box_lid_only != 0);
    const int cap = lid ? nx + 1 : 2 * nx + 2 * imax(ny - 2, 0) + 1;
    B->xref = dalloc(cap); B->yref = dalloc(cap); B->zref = dalloc(cap);
    int m = 1;
#define ADDM(X, Y) do { B->xref[m] = (X); B->yref[m] = (Y); B->zref[m] = 0.0; ++m; } while (0)
    if (lid) {
      for (int i = 0; i < nx; ++i) ADDM(xlo + (double)i * dsx, yhi);
    } else {
      for (int i = 0; i < nx; ++i) ADDM(xlo + (double)i * dsx, ylo);
      for (int i = 0; i < nx; ++i) ADDM(xlo + (double)i * dsx, yhi);
      for (int j = 1; j < ny - 1; ++j) {
        const double yy = ylo + (double)j * dsy;
        ADDM(xlo, yy);
        ADDM(xhi, yy);
      }
    }
#undef ADDM
    Ml = m - 1;
    const double perim = lid ? (xhi - xlo) : 2.0 * ((xhi - xlo) + (yhi - ylo));
    const double ds_eff = perim / (double)Ml;
    dv = ds_eff * h;
    B->wall_tol = (p->box_wall_tol > 0.0) ? p->box_wall_tol : dmax(0.25 * dmin(dsx, dsy), 1.0e-12);
  } else if (p->geometry_type == 2) { /* user-defined pitching NACA, 2D only */
    if (L->dim != 2) return -1;
    const double chord = dmax(B->chord, 1.0e-12), thick = dmax(B->thick, 1.0e-12);
    const int n_half = (p->n_marker > 0) ? imax(p->n_marker / 2, 32)
                                         : imax((int)ceil(1.5 * chord / h), 48);
    const int cap = 2 * n_half + 2;
    B->xref = dalloc(cap); B->yref = dalloc(cap); B->zref = dalloc(cap);
    int m = 1;
    for (int i = 0; i <= n_half; ++i) {
      const double beta = pi * (double)i / (double)n_half;
      const double x = 0.5 * chord * (1.0 - cos(beta));
      const double xc = dmin(dmax(x / chord, 0.0), 1.0);
      const double sx = sqrt(dmax(xc, 0.0));
      B->xref[m] = x;
      B->yref[m] = 5.0 * thick * chord *
                   (0.2969 * sx - 0.1260 * xc - 0.3516 * xc * xc + 0.2843 * xc * xc * xc -
                    0.1036 * xc * xc * xc * xc);
      B->zref[m] = 0.0;
      ++m;
    }
    for (int i = n_half - 1; i >= 1; --i) {
      const double beta = pi * (double)i / (double)n_half;
      const double x = 0.5 * chord * (1.0 - cos(beta));
      const double xc = dmin(dmax(x / chord, 0.0), 1.0);
      const double sx = sqrt(dmax(xc, 0.0));
      B->xref[m] = x;
      B->yref[m] = -(5.0 * thick * chord *
                     (0.2969 * sx - 0.1260 * xc - 0.3516 * xc * xc + 0.2843 * xc * xc * xc -
                      0.1036 * xc * xc * xc * xc));
      B->zref[m] = 0.0;
      ++m;
    }
    Ml = m - 1;
    double perim = 0.0;
    for (int i = 1; i <= Ml; ++i) {
      const int in = (i == Ml) ? 1 : (i + 1);
      const double a = B->xref[in] - B->xref[i], b = B->yref[in] - B->yref[i];
      perim += sqrt(a * a + b * b);
    }
    dv = (perim / (double)Ml) * h;
    B->wall_tol = 0.0;
  } else if (L->dim == 2) { /* circle */
    if (Ml <= 0) {
      Ml = (int)ceil(2.0 * pi * p->R / h);
      Ml = imax(Ml, 16);
    }
    dv = (2.0 * pi * p->R * h) / (double)Ml;
    B->phi = dalloc(Ml + 1);
    B->theta = dalloc(Ml + 1);
    for (int i = 0; i <= Ml; ++i) B->theta[i] = 0.5 * pi;
    for (int i = 1; i <= Ml; ++i) B->phi[i] = 2.0 * pi * (double)(i - 1) / (double)Ml;
    B->wall_tol = 0.0;
  } else { /* sphere: golden spiral */
    const double rd = p->rd;
    const double a1 = pow(p->R - (rd - 0.5) * h, 3), a2 = pow(p->R - (rd + 0.5) * h, 3);
    {
      /* Math::powi<3> is x*x*x; keep that product order */
      const double t1 = p->R - (rd - 0.5) * h, t2 = p->R - (rd + 0.5) * h;
      (void)a1; (void)a2;
      const double b1 = 1.0 * t1 * t1 * t1, b2 = 1.0 * t2 * t2 * t2;
      if (Ml <= 0) {
        const double denom = 3.0 * h * h * h / 4.0 / pi;
        Ml = (int)((b1 - b2) / denom);
        Ml = imax(Ml, 32);
      }
      dv = (b1 - b2) / (3.0 * (double)Ml / 4.0 / pi);
    }
    B->phi = dalloc(Ml + 1);
    B->theta = dalloc(Ml + 1);
    double ph = 0.0;
    for (int mi = 0; mi < Ml; ++mi) {
      const double Hk = -1.0 + 2.0 * (double)mi / ((double)Ml - 1.0);
      const double th = acos(Hk);
      if (mi == 0 || mi == Ml - 1) ph = 0.0;
      else ph = fmod(ph + 3.809 / sqrt((double)Ml) / sqrt(1.0 - Hk * Hk), 2.0 * pi);
      B->phi[mi + 1] = ph;
      B->theta[mi + 1] = th;
    }
    B->wall_tol = 0.0;
  }
  B->n = Ml;
  B->dv = dv;
  B->x = dalloc(Ml); B->y = dalloc(Ml); B->z = dalloc(Ml);
  B->u = dalloc(Ml); B->v = dalloc(Ml); B->w = dalloc(Ml);
  B->fx = dalloc(Ml); B->fy = dalloc(Ml); B->fz = dalloc(Ml);
  B->mx = dalloc(Ml); B->my = dalloc(Ml); B->mz = dalloc(Ml);
  return 0;
}

/* marker position of marker idx (1-based) at time t: the formulas shared by
 * update_lagrangian_marker (IBMarkerDF.cpp:544-605) and gather_marker_state (:875-943) */
static void marker_pos(const orc_level *L, int idx, double t, double *x, double *y, double *z,
                       double *ut, double *vt, double *wt) {
  const orc_ib *B = &L->ib;
  const double z0 = (L->dim == 3) ? B->p.z0 : 0.0;
  *ut = *vt = *wt = 0.0;
  if (B->p.geometry_type == 1) {
    *x = B->xref[idx]; *y = B->yref[idx]; *z = (L->dim == 3) ? B->zref[idx] : 0.0;
  } else if (B->p.geometry_type == 2) {
    user_marker_state(L, idx, t, x, y, z, ut, vt, wt);
    if (L->dim != 3) *z = 0.0;
  } else {
    *x = B->p.x0 + B->p.R * sin(B->theta[idx]) * cos(B->phi[idx]);
    *y = B->p.y0 + B->p.R * sin(B->theta[idx]) * sin(B->phi[idx]);
    *z = (L->dim == 3) ? z0 + B->p.R * cos(B->theta[idx]) : 0.0;
  }
}

/* update_lagrangian_marker, IBMarkerDF.cpp:499-609 (single tile; Redistribute wraps
 * periodic coordinates) */
static void update_lagrangian_marker(orc_level *L, double t) {
  orc_ib *B = &L->ib;
  for (int i = 0; i < B->n; ++i) {
    double x, y, z, ut, vt, wt;
    marker_pos(L, i + 1, t, &x, &y, &z, &ut, &vt, &wt);
    double pos[3] = {x, y, z};
    for (int d = 0; d < L->dim; ++d) {
      if (!L->periodic[d]) continue;
      const double lo = L->plo[d], hi = L->phi[d], Lx = hi - lo;
      while (pos[d] < lo) pos[d] += Lx;
      while (pos[d] >= hi) pos[d] -= Lx;
    }
    B->x[i] = pos[0]; B->y[i] = pos[1]; B->z[i] = pos[2];
    B->mx[i] = ut; B->my[i] = vt; B->mz[i] = wt;
    B->u[i] = B->v[i] = B->w[i] = 0.0;
    B->fx[i] = B->fy[i] = B->fz[i] = 0.0;
  }
}

typedef struct { int ilo, ihi, jlo, jhi, klo, khi; } clipbox;

/* velocity_interpolation_cic, IBMarkerDF.cpp:612-695 (E: 3-comp grown array) */
static void interp_marker(const orc_level *L, int m, const double *E, clipbox cb, int kt,
                          int renorm, double *Up, double *Vp, double *Wp) {
  const orc_ib *B = &L->ib;
  const double *dx = L->dx, *plo = L->plo;
  const double d = (L->dim == 3) ? dx[0] * dx[1] * dx[2] : dx[0] * dx[1];
  const double px = B->x[m], py = B->y[m], pz = B->z[m];
  const double lx = (px - plo[0]) / dx[0];
  const double ly = (py - plo[1]) / dx[1];
  const double lz = (L->dim == 3) ? (pz - plo[2]) / dx[2] : 0.0;
  const int i0 = (int)floor(lx), j0 = (int)floor(ly), k0 = (int)floor(lz);
  double u = 0.0, v = 0.0, w = 0.0, part = 0.0;
  const long s = L->gcells;
  for (int ii = -2; ii < 3; ++ii) {
    const double xi = plo[0] + ((double)(i0 + ii) + 0.5) * dx[0];
    const double tU = orc_delta(xi, px, dx[0], kt);
    for (int jj = -2; jj < 3; ++jj) {
      const double yi = plo[1] + ((double)(j0 + jj) + 0.5) * dx[1];
      const double tV = orc_delta(yi, py, dx[1], kt);
      if (L->dim == 3) {
        for (int kk = -2; kk < 3; ++kk) {
          const double zi = plo[2] + ((double)(k0 + kk) + 0.5) * dx[2];
          const double tW = orc_delta(zi, pz, dx[2], kt);
          const int ip = i0 + ii, jp = j0 + jj, kp = k0 + kk;
          if (ip < cb.ilo || ip > cb.ihi || jp < cb.jlo || jp > cb.jhi || kp < cb.klo || kp > cb.khi)
            continue;
          const double dvl = tU * tV * tW;
          const long e = IX(L, ip, jp, kp);
          part += dvl * d;
          u += dvl * E[e] * d;
          v += dvl * E[e + s] * d;
          w += dvl * E[e + 2 * s] * d;
        }
      } else {
        const int ip = i0 + ii, jp = j0 + jj;
        if (ip < cb.ilo || ip > cb.ihi || jp < cb.jlo || jp > cb.jhi) continue;
        const double dvl = tU * tV;
        const long e = IX(L, ip, jp, 0);
        part += dvl * d;
        u += dvl * E[e] * d;
        v += dvl * E[e + s] * d;
        w += 0.0;
      }
    }
  }
  if (renorm && part > 0.0) { u /= part; v /= part; w /= part; }
  *Up = u; *Vp = v; *Wp = w;
}

/* compute_lagrangian_force_explicit, IBMarkerDF.cpp:741-873 */
static void force_explicit(orc_level *L, double dt, double t) {
  orc_ib *B = &L->ib;
  const ilbm_ib_case *p = &B->p;
  const double relax = dmax(0.0, dmin(1.0, p->mdf_relax));
  const int diag = (p->coupling_method == 2);
  const double diag_eps = dmax(p->explicit_diag_eps, 1.0e-30);
  const double *dx = L->dx, *plo = L->plo;
  const int kt = B->kernel;
  (void)t;
  for (int i = 0; i < B->n; ++i) {
    double Ux = 0.0, Uy = 0.0, Uz = 0.0;
    const double px = B->x[i], py = B->y[i], pz = (L->dim == 3) ? B->z[i] : 0.0;
    if (p->geometry_type == 2) { Ux = B->mx[i]; Uy = B->my[i]; Uz = B->mz[i]; }
    else rigid_target(L, px, py, pz, &Ux, &Uy, &Uz);
    double denom = dt;
    if (diag) {
      const double dV = (L->dim == 3) ? dx[0] * dx[1] * dx[2] : dx[0] * dx[1];
      const double lx = (px - plo[0]) / dx[0], ly = (py - plo[1]) / dx[1];
      const double lz = (L->dim == 3) ? (pz - plo[2]) / dx[2] : 0.0;
      const int i0 = (int)floor(lx), j0 = (int)floor(ly), k0 = (int)floor(lz);
      double sum2 = 0.0;
      for (int ii = -2; ii < 3; ++ii) {
        const int ip = i0 + ii;
        if (ip < 0 || ip > L->n[0] - 1) continue;
        const double xi = plo[0] + ((double)ip + 0.5) * dx[0];
        const double tU = orc_delta(xi, px, dx[0], kt);
        for (int jj = -2; jj < 3; ++jj) {
          const int jp = j0 + jj;
          if (jp < 0 || jp > L->n[1] - 1) continue;
          const double yi = plo[1] + ((double)jp + 0.5) * dx[1];
          const double tV = orc_delta(yi, py, dx[1], kt);
          if (L->dim == 3) {
            for (int kk = -2; kk < 3; ++kk) {
              const int kp = k0 + kk;
              if (kp < 0 || kp > L->n[2] - 1) continue;
              const double zi = plo[2] + ((double)kp + 0.5) * dx[2];
              const double tW = orc_delta(zi, pz, dx[2], kt);
              const double dvl = tU * tV * tW;
              sum2 += dvl * dvl * dV;
            }
          } else {
            const double dvl = tU * tV;
            sum2 += dvl * dvl * dV;
          }
        }
      }
      const double mkk = B->dv * sum2;
      denom = dt * dmax(mkk, diag_eps);
    }
    B->fx[i] += relax * (Ux - B->u[i]) / denom;
    B->fy[i] += relax * (Uy - B->v[i]) / denom;
    B->fz[i] += relax * (Uz - B->w[i]) / denom;
  }
}

/* lu_factorize / lu_solve, IBMarkerDF.cpp:1015-1079 */
static int lu_factorize(double *a, int *piv, int n, double tiny) {
  for (int k = 0; k < n; ++k) {
    int p = k;
    double maxv = fabs(a[(long)k * n + k]);
    for (int i = k + 1; i < n; ++i) {
      const double v = fabs(a[(long)i * n + k]);
      if (v > maxv) { maxv = v; p = i; }
    }
    if (maxv <= tiny) return 0;
    piv[k] = p;
    if (p != k)
      for (int j = 0; j < n; ++j) {
        double t = a[(long)k * n + j];
        a[(long)k * n + j] = a[(long)p * n + j];
        a[(long)p * n + j] = t;
      }
    const double akk = a[(long)k * n + k];
    for (int i = k + 1; i < n; ++i) {
      a[(long)i * n + k] /= akk;
      const double lik = a[(long)i * n + k];
      for (int j = k + 1; j < n; ++j) a[(long)i * n + j] -= lik * a[(long)k * n + j];
    }
  }
  return 1;
}
static void lu_solve(const double *a, const int *piv, const double *rhs, double *x, int n) {
  for (int i = 0; i < n; ++i) x[i] = rhs[i];
  for (int k = 0; k < n; ++k) {
    const int p = piv[k];
    if (p != k) { double t = x[k]; x[k] = x[p]; x[p] = t; }
  }
  for (int i = 1; i < n; ++i) {
    double sum = x[i];
    for (int j = 0; j < i; ++j) sum -= a[(long)i * n + j] * x[j];
    x[i] = sum;
  }
  for (int i = n - 1; i >= 0; --i) {
    double sum = x[i];
    for (int j = i + 1; j < n; ++j) sum -= a[(long)i * n + j] * x[j];
    x[i] = sum / a[(long)i * n + i];
  }
}

/* build_ivc_operator, IBMarkerDF.cpp:1081-1142 */
static void build_ivc(orc_level *L, const double *xg, const double *yg, const double *zg) {
  orc_ib *B = &L->ib;
  const int n = B->n;
  B->ivc_ready = 0;
  B->ivc_n = n;
  free(B->lu); free(B->piv); free(B->xc); free(B->yc); free(B->zc);
  B->lu = dalloc((long)n * n);
  B->piv = (int *)calloc((size_t)n, sizeof(int));
  const int kt = B->kernel;
  for (int i = 0; i < n; ++i)
    for (int j = i; j < n; ++j) {
      const double sx = orc_overlap_1d(xg[i], xg[j], L->dx[0], kt, L->plo[0], 0, L->n[0] - 1);
      const double sy = orc_overlap_1d(yg[i], yg[j], L->dx[1], kt, L->plo[1], 0, L->n[1] - 1);
      const double sz = (L->dim == 3)
                            ? orc_overlap_1d(zg[i], zg[j], L->dx[2], kt, L->plo[2], 0, L->n[2] - 1)
                            : 1.0;
      double val = B->dv * sx * sy * sz;
      if (i == j) val += B->p.ivc_diag_reg;
      B->lu[(long)i * n + j] = val;
      B->lu[(long)j * n + i] = val;
    }
  const double tiny = dmax(B->p.ivc_diag_reg * 1.0e-4, 1.0e-30);
  B->ivc_ready = lu_factorize(B->lu, B->piv, n, tiny);
  B->xc = dalloc(n); B->yc = dalloc(n); B->zc = dalloc(n);
  memcpy(B->xc, xg, sizeof(double) * n);
  memcpy(B->yc, yg, sizeof(double) * n);
  memcpy(B->zc, zg, sizeof(double) * n);
}

/* compute_lagrangian_force_ivc, IBMarkerDF.cpp:1144-1328 (one rank) */
static void force_ivc(orc_level *L, double dt, double t) {
  orc_ib *B = &L->ib;
  const int n = B->n;
  if (n <= 0) return;
  double *xg = dalloc(n), *yg = dalloc(n), *zg = dalloc(n);
  for (int i = 0; i < n; ++i) {
    double ut, vt, wt;
    marker_pos(L, i + 1, t, &xg[i], &yg[i], &zg[i], &ut, &vt, &wt);
  }
  int changed = (B->xc == NULL) || (B->ivc_n != n);
  if (!changed)
    for (int i = 0; i < n; ++i)
      if (fabs(xg[i] - B->xc[i]) > 1.0e-12 || fabs(yg[i] - B->yc[i]) > 1.0e-12 ||
          fabs(zg[i] - B->zc[i]) > 1.0e-12) { changed = 1; break; }
  if (!B->ivc_ready || B->ivc_n != n || B->p.ivc_rebuild_matrix > 0 || changed)
    build_ivc(L, xg, yg, zg);
  if (!B->ivc_ready) {
    free(xg); free(yg); free(zg);
    force_explicit(L, dt, t);
    return;
  }
  double *bx = dalloc(n), *by = dalloc(n), *bz = dalloc(n);
  double *sx = dalloc(n), *sy = dalloc(n), *sz = dalloc(n);
  for (int i = 0; i < n; ++i) {
    double Ux = 0.0, Uy = 0.0, Uz = 0.0;
    if (B->p.geometry_type == 2) {
      double px, py, pz;
      user_marker_state(L, i + 1, t, &px, &py, &pz, &Ux, &Uy, &Uz);
    } else {
      rigid_target(L, xg[i], yg[i], zg[i], &Ux, &Uy, &Uz);
    }
    bx[i] = (Ux - B->u[i]) / dt;
    by[i] = (Uy - B->v[i]) / dt;
    bz[i] = (Uz - B->w[i]) / dt;
  }
  lu_solve(B->lu, B->piv, bx, sx, n);
  lu_solve(B->lu, B->piv, by, sy, n);
  lu_solve(B->lu, B->piv, bz, sz, n);
  for (int i = 0; i < n; ++i) { B->fx[i] += sx[i]; B->fy[i] += sy[i]; B->fz[i] += sz[i]; }
  free(xg); free(yg); free(zg); free(bx); free(by); free(bz); free(sx); free(sy); free(sz);
}

/* Order in which markers are spread (test aid, process-wide): 0 = marker
 * order, as the reference's loop over particles; 1 = reversed.  The FP64
 * atomic spreading of the device path sums in an unspecified order, so its
 * parity tests measure how far the reference's own result moves when only
 * this order changes and allow the device that much. */
static int g_spread_reverse = 0;
void orc_set_spread_order(int reverse) { g_spread_reverse = reverse ? 1 : 0; }

/* force_spreading_cic + force_spreading, IBMarkerDF.cpp:1331-1512 (E: grown array) */
static void spread(orc_level *L, double *E, clipbox cb) {
  orc_ib *B = &L->ib;
  const double *dx = L->dx, *plo = L->plo;
  const int kt = B->kernel;
  const int renorm = (B->p.renormalize_delta != 0);
  const long s = L->gcells;
  const double d = (L->dim == 3) ? dx[0] * dx[1] * dx[2] : dx[0] * dx[1];
  const double z0 = (L->dim == 3) ? B->p.z0 : 0.0;
  for (int mm = 0; mm < B->n; ++mm) {
    const int m = g_spread_reverse ? B->n - 1 - mm : mm;
    const double fx = B->fx[m] * B->dv, fy = B->fy[m] * B->dv, fz = B->fz[m] * B->dv;
    const double px = B->x[m], py = B->y[m], pz = (L->dim == 3) ? B->z[m] : 0.0;
    const double rx = px - B->p.x0, ry = py - B->p.y0, rz = (L->dim == 3) ? pz - z0 : 0.0;
    B->mx[m] = ry * fz - rz * fy;
    B->my[m] = rz * fx - rx * fz;
    B->mz[m] = rx * fy - ry * fx;
    const double lx = (px - plo[0]) / dx[0], ly = (py - plo[1]) / dx[1];
    const double lz = (L->dim == 3) ? (pz - plo[2]) / dx[2] : 0.0;
    const int i0 = (int)floor(lx), j0 = (int)floor(ly), k0 = (int)floor(lz);
    double part = 0.0;
    for (int pass = 0; pass < 2; ++pass) {
      double scale = 1.0;
      if (pass == 1 && renorm && part > 0.0) scale = 1.0 / part;
      for (int ii = -2; ii < 3; ++ii) {
        const double xi = plo[0] + ((double)(i0 + ii) + 0.5) * dx[0];
        const double tU = orc_delta(xi, px, dx[0], kt);
        for (int jj = -2; jj < 3; ++jj) {
          const double yi = plo[1] + ((double)(j0 + jj) + 0.5) * dx[1];
          const double tV = orc_delta(yi, py, dx[1], kt);
          if (L->dim == 3) {
            for (int kk = -2; kk < 3; ++kk) {
              const double zi = plo[2] + ((double)(k0 + kk) + 0.5) * dx[2];
              const double tW = orc_delta(zi, pz, dx[2], kt);
              const int ip = i0 + ii, jp = j0 + jj, kp = k0 + kk;
              if (ip < cb.ilo || ip > cb.ihi || jp < cb.jlo || jp > cb.jhi || kp < cb.klo ||
                  kp > cb.khi)
                continue;
              if (pass == 0) { part += tU * tV * tW * d; continue; }
              const double dvl = (tU * tV * tW) * scale;
              const long e = IX(L, ip, jp, kp);
              E[e] += dvl * fx;
              E[e + s] += dvl * fy;
              E[e + 2 * s] += dvl * fz;
            }
          } else {
            const int ip = i0 + ii, jp = j0 + jj;
            if (ip < cb.ilo || ip > cb.ihi || jp < cb.jlo || jp > cb.jhi) continue;
            if (pass == 0) { part += tU * tV * d; continue; }
            const double dvl = (tU * tV) * scale;
            const long e = IX(L, ip, jp, 0);
            E[e] += dvl * fx;
            E[e + s] += dvl * fy;
          }
        }
      }
    }
  }
}

/* MultiFab::SumBoundary(periodicity) restricted to the grown region of ng_e */
static void sum_boundary(const orc_level *L, double *E, int nc, int ng_e) {
  const int kz0 = (L->dim == 3) ? -ng_e : 0, kz1 = (L->dim == 3) ? L->n[2] + ng_e : 1;
  for (int k = kz0; k < kz1; ++k)
    for (int j = -ng_e; j < L->n[1] + ng_e; ++j)
      for (int i = -ng_e; i < L->n[0] + ng_e; ++i) {
        if (in_domain(L, i, j, k)) continue;
        int iv[3] = {i, j, k}, w[3];
        if (wrap_cell(L, iv, w) != 0) continue;
        const long gi = IX(L, i, j, k), wi = IX(L, w[0], w[1], w[2]);
        for (int n = 0; n < nc; ++n) E[wi + n * L->gcells] += E[gi + n * L->gcells];
      }
}

/* FillBoundary on a field that lives on the grown region of ng_e */
static void fill_boundary_ng(const orc_level *L, double *a, int nc, int ng_e) {
  const int kz0 = (L->dim == 3) ? -ng_e : 0, kz1 = (L->dim == 3) ? L->n[2] + ng_e : 1;
  for (int k = kz0; k < kz1; ++k)
    for (int j = -ng_e; j < L->n[1] + ng_e; ++j)
      for (int i = -ng_e; i < L->n[0] + ng_e; ++i) {
        if (in_domain(L, i, j, k)) continue;
        int iv[3] = {i, j, k}, w[3];
        if (wrap_cell(L, iv, w) != 0) continue;
        const long gi = IX(L, i, j, k), wi = IX(L, w[0], w[1], w[2]);
        for (int n = 0; n < nc; ++n) a[gi + n * L->gcells] = a[wi + n * L->gcells];
      }
}

/* update_forcing, IBMarkerDF.cpp:1522-1917.  smS: FillPatched macro (6 comps, grown);
 * fcc: force output (3 comps, grown), valid cells written. */
static void ib_update_forcing(orc_level *L, const double *smS, double *fcc, double dt,
                              double t) {
  orc_ib *B = &L->ib;
  const int ngE = 2;
  const long s = L->gcells;
  double *EV = dalloc(3 * s), *EFI = dalloc(3 * s), *EFT = dalloc(3 * s);
  const int kz0 = (L->dim == 3) ? -ngE : 0, kz1 = (L->dim == 3) ? L->n[2] + ngE : 1;
  for (int k = kz0; k < kz1; ++k)
    for (int j = -ngE; j < L->n[1] + ngE; ++j)
      for (int i = -ngE; i < L->n[0] + ngE; ++i) {
        const long e = IX(L, i, j, k);
        EV[e] = smS[e + s];
        EV[e + s] = smS[e + 2 * s];
        EV[e + 2 * s] = (L->dim == 3) ? smS[e + 3 * s] : 0.0;
      }
  fill_boundary_ng(L, EV, 3, ngE);
  B->fsum[0] = B->fsum[1] = B->fsum[2] = 0.0;
  const int use_ivc = (B->p.coupling_method == 1);
  const int nloop = use_ivc ? 1 : imax(B->p.loop_ns, 1);
  clipbox cbE = {-ngE, L->n[0] - 1 + ngE, -ngE, L->n[1] - 1 + ngE, 0, 0};
  if (L->dim == 3) { cbE.klo = -ngE; cbE.khi = L->n[2] - 1 + ngE; }
  const int renorm_i = (B->p.renormalize_delta != 0) && !use_ivc;
  for (int it = 0; it < nloop; ++it) {
    memset(EFI, 0, sizeof(double) * 3 * s);
    update_lagrangian_marker(L, t);
    fill_boundary_ng(L, EV, 3, ngE); /* velocity_interpolation's FillBoundary, :700-702 */
    for (int m = 0; m < B->n; ++m) {
      double Up, Vp, Wp;
      interp_marker(L, m, EV, cbE, B->kernel, renorm_i, &Up, &Vp, &Wp);
      B->u[m] += Up; B->v[m] += Vp; B->w[m] += Wp;
    }
    if (use_ivc) force_ivc(L, dt, t);
    else force_explicit(L, dt, t);
    spread(L, EFI, cbE);
    sum_boundary(L, EFI, 3, ngE);
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int m = 0; m < B->n; ++m) {
      sx += B->fx[m] * B->dv;
      sy += B->fy[m] * B->dv;
      sz += B->fz[m] * B->dv;
    }
    B->fsum[0] += sx; B->fsum[1] += sy; B->fsum[2] += sz;
    /* velocity_correction (Saxpy, valid cells) and EulerForceTotal += EulerForceIter */
    const int vk0 = 0, vk1 = (L->dim == 3) ? L->n[2] : 1;
    for (int k = vk0; k < vk1; ++k)
      for (int j = 0; j < L->n[1]; ++j)
        for (int i = 0; i < L->n[0]; ++i) {
          const long e = IX(L, i, j, k);
          for (int n = 0; n < 3; ++n) EV[e + n * s] += dt * EFI[e + n * s];
        }
    for (int k = vk0; k < vk1; ++k)
      for (int j = 0; j < L->n[1]; ++j)
        for (int i = 0; i < L->n[0]; ++i) {
          const long e = IX(L, i, j, k);
          for (int n = 0; n < 3; ++n) EFT[e + n * s] += EFI[e + n * s];
        }
  }
  const int vk1 = (L->dim == 3) ? L->n[2] : 1;
  for (int k = 0; k < vk1; ++k)
    for (int j = 0; j < L->n[1]; ++j)
      for (int i = 0; i < L->n[0]; ++i) {
        const long e = IX(L, i, j, k);
        for (int n = 0; n < 3; ++n) fcc[e + n * s] = dt * smS[e] * EFT[e + n * s];
      }
  fill_boundary(L, fcc, 3);
  free(EV); free(EFI); free(EFT);
}

/* ------------------------------------------------------------------------ */
/* level step, Source/Core/AdvanceLBMAtLevel.cpp:20-394                      */
/* ------------------------------------------------------------------------ */
static void compute_ib_force(orc_level *L);

static void level_step(orc_level *L) {
  double *t;
  t = L->f_new; L->f_new = L->f_old; L->f_old = t;       /* :23 */
  t = L->mac_new; L->mac_new = L->mac_old; L->mac_old = t; /* :24 */
  const int Q = L->Q;
  const long s = L->gcells;
  double *fcc = dalloc(3 * s); /* fx_cc, fy_cc, fz_cc, :43-56 */
  if (L->c.use_prescribed_force)
    for (long e = 0; e < s; ++e)
      for (int n = 0; n < 3; ++n) fcc[e + n * s] = L->c.prescribed_force[n];
  double *sfS = dalloc((long)Q * s), *smS = dalloc(6 * s);
  fill_patch(L, sfS, L->f_old, Q, 1);   /* :59 */
  fill_patch(L, smS, L->mac_old, 6, 0); /* :60 */
  if (L->use_ib) ib_update_forcing(L, smS, fcc, L->dt, L->time); /* :83-93 */
  const int vk1 = (L->dim == 3) ? L->n[2] : 1;
  for (int k = 0; k < vk1; ++k)
    for (int j = 0; j < L->n[1]; ++j)
      for (int i = 0; i < L->n[0]; ++i) {
        const long e = IX(L, i, j, k);
        for (int n = 0; n < 3; ++n) {
          if (L->use_ib) L->forcing[e + n * s] = fcc[e + n * s]; /* :122-153 */
          L->last_fx[e + n * s] = fcc[e + n * s];
        }
      }
  fill_boundary(L, fcc, 3); /* :192-194 */
  /* collide, :207-240 */
  for (int k = 0; k < vk1; ++k)
    for (int j = 0; j < L->n[1]; ++j)
      for (int i = 0; i < L->n[0]; ++i) {
        const long e = IX(L, i, j, k);
        const double rho = smS[e], u = smS[e + s], v = smS[e + 2 * s], w = smS[e + 3 * s];
        double feq[ILBM_MAX_Q];
        for (int q = 0; q < Q; ++q) feq[q] = orc_feq(L, L->w[q], L->cx[q], L->cy[q], L->cz[q], rho, u, v, w);
        orc_collide_forced(L, sfS + e, s, feq, L->tau, u, v, w, fcc[e], fcc[e + s], fcc[e + 2 * s]);
      }
  fill_boundary(L, sfS, Q); /* :244 */
  /* halfway bounce-back ghosts, :272-373 */
  {
    const int kz0 = (L->dim == 3) ? -L->ng : 0, kz1 = (L->dim == 3) ? L->n[2] + L->ng : 1;
    for (int k = kz0; k < kz1; ++k)
      for (int j = -L->ng; j < L->n[1] + L->ng; ++j)
        for (int i = -L->ng; i < L->n[0] + L->ng; ++i) {
          if (in_domain(L, i, j, k)) continue;
          int iv[3] = {i, j, k}, has_bb = 0, unsup = 0;
          for (int d = 0; d < L->dim; ++d) {
            if (iv[d] < 0) { if (L->bclo[d] == BC_USER_1) has_bb = 1; else unsup = 1; }
            else if (iv[d] > L->n[d] - 1) { if (L->bchi[d] == BC_USER_1) has_bb = 1; else unsup = 1; }
          }
          if (!has_bb || unsup) continue;
          for (int q = 0; q < Q; ++q) {
            const int it = i + (int)L->cx[q], jt = j + (int)L->cy[q];
            const int kt = (L->dim == 3) ? k + (int)L->cz[q] : k;
            if (!in_domain(L, it, jt, kt)) continue;
            const int rx = -(int)L->cx[q], ry = -(int)L->cy[q], rz = (L->dim == 3) ? -(int)L->cz[q] : 0;
            int qr = q;
            for (int p = 0; p < Q; ++p)
              if ((int)L->cx[p] == rx && (int)L->cy[p] == ry && (int)L->cz[p] == rz) { qr = p; break; }
            sfS[IX(L, i, j, k) + q * s] = sfS[IX(L, it, jt, kt) + qr * s];
          }
        }
  }
  /* stream + macro, :376-386 */
  for (int k = 0; k < vk1; ++k)
    for (int j = 0; j < L->n[1]; ++j)
      for (int i = 0; i < L->n[0]; ++i) {
        const long e = IX(L, i, j, k);
        for (int q = 0; q < Q; ++q) {
          const int ip = i - (int)L->cx[q], jp = j - (int)L->cy[q];
          const int kp = (L->dim == 3) ? k - (int)L->cz[q] : k;
          L->f_new[e + q * s] = sfS[IX(L, ip, jp, kp) + q * s];
        }
      }
  for (int k = 0; k < vk1; ++k)
    for (int j = 0; j < L->n[1]; ++j)
      for (int i = 0; i < L->n[0]; ++i) {
        const long e = IX(L, i, j, k);
        double r = 0, m1 = 0, m2 = 0, m3 = 0;
        for (int q = 0; q < Q; ++q) {
          const double fq = L->f_new[e + q * s];
          r += fq;
          m1 += L->cx[q] * fq;
          m2 += L->cy[q] * fq;
          m3 += L->cz[q] * fq;
        }
        L->mac_new[e] = r;
        L->mac_new[e + s] = (m1 + 0.5 * fcc[e]) / r;
        L->mac_new[e + 2 * s] = (m2 + 0.5 * fcc[e + s]) / r;
        L->mac_new[e + 3 * s] = (m3 + 0.5 * fcc[e + 2 * s]) / r;
      }
  free(fcc); free(sfS); free(smS);
}

/* ComputeIBForce, Source/Core/AmrCoreLBM.cpp:456-631 (no file output) */
static void compute_ib_force(orc_level *L) {
  if (!L->use_ib) return;
  const long s = L->gcells;
  double Fs[3] = {0, 0, 0};
  const int vk1 = (L->dim == 3) ? L->n[2] : 1;
  for (int n = 0; n < 3; ++n) {
    double acc = 0.0;
    for (int k = 0; k < vk1; ++k)
      for (int j = 0; j < L->n[1]; ++j)
        for (int i = 0; i < L->n[0]; ++i) acc += L->forcing[IX(L, i, j, k) + n * s];
    Fs[n] = acc;
  }
  if (L->dim != 3) Fs[2] = 0.0;
  double dV = L->dx[0];
  dV *= L->dx[1];
  if (L->dim == 3) dV *= L->dx[2];
  double Fe[3], Fm[3], Fme[3], Fb[3], Ftc[3];
  for (int n = 0; n < 3; ++n) {
    Fe[n] = -(Fs[n] * dV) / L->dt;
    Fm[n] = -L->ib.fsum[n];
    Fme[n] = Fe[n];
    Fb[n] = Fe[n];
    if (L->ib.p.force_eval_method == 2) Fb[n] = Fm[n];
    else if (L->ib.p.force_eval_method == 0) Fb[n] = Fme[n];
    Ftc[n] = Fb[n];
    if (L->have_prev) Ftc[n] = 0.5 * (L->prev[n] + Fb[n]);
    L->prev[n] = Fb[n];
  }
  L->have_prev = 1;
  const double U = L->ib.p.U0, D = 2.0 * L->ib.p.R;
  const double denom = (L->dim == 3) ? 0.5 * 1.0 * U * U * (3.14159265358979323846 * L->ib.p.R * L->ib.p.R)
                                     : 0.5 * 1.0 * U * U * D;
  for (int n = 0; n < 3; ++n) {
    L->rec[n] = Ftc[n];
    L->rec[6 + n] = Fb[n];
    L->rec[9 + n] = Fe[n];
    L->rec[12 + n] = Fm[n];
    L->rec[15 + n] = Fme[n];
  }
  L->rec[3] = L->rec[4] = L->rec[5] = 0.0;
  if (denom > 0.0) {
    L->rec[3] = Ftc[0] / denom;
    L->rec[4] = Ftc[1] / denom;
    if (L->dim == 3) L->rec[5] = Ftc[2] / denom;
  }
}

/* ------------------------------------------------------------------------ */
/* C API (mirrors oracle/ref_driver.cpp)                                    */
/* ------------------------------------------------------------------------ */
static void copy_valid(const orc_level *L, const double *src, int nc, double *dst, int to_grown) {
  const int vk1 = (L->dim == 3) ? L->n[2] : 1;
  const long nv = (long)L->n[0] * L->n[1] * vk1;
  long idx = 0;
  for (int k = 0; k < vk1; ++k)
    for (int j = 0; j < L->n[1]; ++j)
      for (int i = 0; i < L->n[0]; ++i, ++idx) {
        const long e = IX(L, i, j, k);
        for (int c = 0; c < nc; ++c) {
          if (to_grown) dst[e + c * L->gcells] = src[idx + c * nv];
          else dst[idx + c * nv] = src[e + c * L->gcells];
        }
      }
}

void *orc_create(const ilbm_case *c) {
  if (c->dim != 2 && c->dim != 3) return NULL;
  if (c->q <= 0 || c->q > ILBM_MAX_Q) return NULL;
  orc_level *L = (orc_level *)calloc(1, sizeof(orc_level));
  L->c = *c;
  L->dim = c->dim;
  L->Q = c->q;
  L->ng = c->nghost > 0 ? c->nghost : 3;
  L->ngz = (c->dim == 3) ? L->ng : 0;
  for (int d = 0; d < 3; ++d) {
    L->n[d] = (d < c->dim) ? c->n_cell[d] : 1;
    L->gn[d] = (d < c->dim) ? L->n[d] + 2 * L->ng : 1;
    L->plo[d] = c->prob_lo[d];
    L->phi[d] = c->prob_hi[d];
    L->dx[d] = (d < c->dim) ? (c->prob_hi[d] - c->prob_lo[d]) / (double)c->n_cell[d] : 0.0;
    L->periodic[d] = (d < c->dim) ? c->periodic[d] : 0;
  }
  L->gcells = (long)L->gn[0] * L->gn[1] * L->gn[2];
  for (int q = 0; q < L->Q; ++q) {
    L->w[q] = c->wis[q] / c->wim[q];
    L->cx[q] = c->cx[q];
    L->cy[q] = c->cy[q];
    L->cz[q] = c->cz[q];
  }
  int allp = 1;
  for (int d = 0; d < c->dim; ++d) allp = allp && c->periodic[d];
  for (int d = 0; d < 3; ++d) {
    if (!allp && d < c->dim) {
      L->bclo[d] = c->bc_lo[d]; L->bchi[d] = c->bc_hi[d];
      L->lo_rho[d] = c->bc_lo_rho[d]; L->lo_ux[d] = c->bc_lo_ux[d];
      L->lo_uy[d] = c->bc_lo_uy[d]; L->lo_uz[d] = c->bc_lo_uz[d];
      L->hi_rho[d] = c->bc_hi_rho[d]; L->hi_ux[d] = c->bc_hi_ux[d];
      L->hi_uy[d] = c->bc_hi_uy[d]; L->hi_uz[d] = c->bc_hi_uz[d];
    } else {
      L->bclo[d] = L->bchi[d] = BC_INT_DIR;
    }
  }
  L->tau = 3.0 * c->nu / L->dx[0] + 0.5;
  L->dt = L->dx[0];
  L->f_new = dalloc((long)L->Q * L->gcells);
  L->f_old = dalloc((long)L->Q * L->gcells);
  L->mac_new = dalloc(6 * L->gcells);
  L->mac_old = dalloc(6 * L->gcells);
  L->forcing = dalloc(3 * L->gcells);
  L->last_fx = dalloc(3 * L->gcells);
  return L;
}

static void free_ib(orc_ib *B) {
  free(B->x); free(B->y); free(B->z); free(B->u); free(B->v); free(B->w);
  free(B->fx); free(B->fy); free(B->fz); free(B->mx); free(B->my); free(B->mz);
  free(B->phi); free(B->theta); free(B->xref); free(B->yref); free(B->zref);
  free(B->lu); free(B->piv); free(B->xc); free(B->yc); free(B->zc);
}

void orc_destroy(void *h) {
  orc_level *L = (orc_level *)h;
  if (!L) return;
  free(L->f_new); free(L->f_old); free(L->mac_new); free(L->mac_old);
  free(L->forcing); free(L->last_fx);
  free_ib(&L->ib);
  free(L);
}

int orc_set_macro(void *h, const double *m4) {
  orc_level *L = (orc_level *)h;
  copy_valid(L, m4, 4, L->mac_new, 1);
  memcpy(L->mac_old, L->mac_new, sizeof(double) * 6 * L->gcells);
  return 0;
}
/* InitEquilibrium, AmrCoreLBM.cpp:2117-2164 (valid cells; ghosts are refilled every step) */
int orc_init_equilibrium(void *h) {
  orc_level *L = (orc_level *)h;
  const long s = L->gcells;
  for (long e = 0; e < s; ++e) {
    const double r = dmax(L->mac_new[e], 1.e-12);
    const double u0 = L->mac_new[e + s], v0 = L->mac_new[e + 2 * s], w0 = L->mac_new[e + 3 * s];
    const double u2 = u0 * u0 + v0 * v0 + w0 * w0;
    for (int q = 0; q < L->Q; ++q) {
      const double cu = L->cx[q] * u0 + L->cy[q] * v0 + L->cz[q] * w0;
      const double feq = L->w[q] * r * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * u2);
      L->f_new[e + q * s] = feq;
      L->f_old[e + q * s] = feq;
    }
  }
  memcpy(L->mac_old, L->mac_new, sizeof(double) * 6 * s);
  return 0;
}
int orc_set_f(void *h, const double *f) { orc_level *L = (orc_level *)h; copy_valid(L, f, L->Q, L->f_new, 1); return 0; }
int orc_get_f(void *h, double *f) { orc_level *L = (orc_level *)h; copy_valid(L, L->f_new, L->Q, f, 0); return 0; }
int orc_get_macro(void *h, double *m4) { orc_level *L = (orc_level *)h; copy_valid(L, L->mac_new, 4, m4, 0); return 0; }
int orc_get_force(void *h, double *f3) { orc_level *L = (orc_level *)h; copy_valid(L, L->last_fx, 3, f3, 0); return 0; }
int orc_set_forcing(void *h, const double *f3) { orc_level *L = (orc_level *)h; copy_valid(L, f3, 3, L->forcing, 1); return 0; }

/* FillPatch of the current populations / macros onto the grown box (for tests of
 * caller-filled ghost mode).  out: [comp][grown k][grown j][grown i]. */
int orc_fill_patch_f(void *h, double *out) {
  orc_level *L = (orc_level *)h;
  memset(out, 0, sizeof(double) * L->Q * L->gcells);
  fill_patch(L, out, L->f_new, L->Q, 1);
  return 0;
}
int orc_fill_patch_macro(void *h, double *out) {
  orc_level *L = (orc_level *)h;
  memset(out, 0, sizeof(double) * 6 * L->gcells);
  fill_patch(L, out, L->mac_new, 6, 0);
  return 0;
}
long orc_grown_cells(void *h) { return ((orc_level *)h)->gcells; }

/* airfoil parameters (defaults: IBMUserDefinedGeometry.H:14-20) */
static double g_af[7] = {20.0, 0.12, 0.0, 0.2617993877991494, 0.0015, 0.0, 0.0};
void orc_set_airfoil(const double *p7) { for (int i = 0; i < 7; ++i) g_af[i] = p7[i]; }

int orc_ib_create(void *h, const ilbm_ib_case *ib) {
  orc_level *L = (orc_level *)h;
  free_ib(&L->ib);
  memset(&L->ib, 0, sizeof(orc_ib));
  L->ib.p = *ib;
  L->ib.kernel = delta_kernel(ib->delta_type);
  L->ib.chord = g_af[0]; L->ib.thick = g_af[1]; L->ib.pitch_mean = g_af[2];
  L->ib.pitch_amp = g_af[3]; L->ib.pitch_freq = g_af[4]; L->ib.pitch_phase = g_af[5];
  L->ib.pivot_x = g_af[6];
  if (ib->geometry_type == 1) {
    if (L->ib.p.box_xhi <= L->ib.p.box_xlo) { L->ib.p.box_xlo = L->plo[0]; L->ib.p.box_xhi = L->phi[0]; }
    if (L->ib.p.box_yhi <= L->ib.p.box_ylo) { L->ib.p.box_ylo = L->plo[1]; L->ib.p.box_yhi = L->phi[1]; }
  }
  if (build_markers(L) != 0) return -1;
  update_lagrangian_marker(L, 0.0);
  L->use_ib = 1;
  memset(L->forcing, 0, sizeof(double) * 3 * L->gcells);
  L->have_prev = 0;
  return 0;
}
long orc_ib_num_markers(void *h) { return ((orc_level *)h)->ib.n; }
double orc_ib_dv(void *h) { return ((orc_level *)h)->ib.dv; }
int orc_ib_marker_force_sum(void *h, double *o3) {
  orc_level *L = (orc_level *)h;
  for (int n = 0; n < 3; ++n) o3[n] = L->ib.fsum[n];
  return 0;
}
/* positions + last interpolated velocity: [n][6] */
int orc_ib_marker_state(void *h, double *o6) {
  orc_level *L = (orc_level *)h;
  for (int m = 0; m < L->ib.n; ++m) {
    o6[m * 6 + 0] = L->ib.x[m]; o6[m * 6 + 1] = L->ib.y[m]; o6[m * 6 + 2] = L->ib.z[m];
    o6[m * 6 + 3] = L->ib.u[m]; o6[m * 6 + 4] = L->ib.v[m]; o6[m * 6 + 5] = L->ib.w[m];
  }
  return 0;
}
/* marker forces of the last iteration: [n][3] */
int orc_ib_marker_force(void *h, double *o3) {
  orc_level *L = (orc_level *)h;
  for (int m = 0; m < L->ib.n; ++m) {
    o3[m * 3 + 0] = L->ib.fx[m]; o3[m * 3 + 1] = L->ib.fy[m]; o3[m * 3 + 2] = L->ib.fz[m];
  }
  return 0;
}

int orc_step(void *h, int nsteps) {
  orc_level *L = (orc_level *)h;
  for (int s = 0; s < nsteps; ++s) {
    level_step(L);
    L->time += L->dt;
    L->step += 1;
    compute_ib_force(L);
  }
  return 0;
}
double orc_time(void *h) { return ((orc_level *)h)->time; }
double orc_tau(void *h) { return ((orc_level *)h)->tau; }
int orc_force_record(void *h, double *out) {
  orc_level *L = (orc_level *)h;
  for (int n = 0; n < ILBM_FORCE_REC; ++n) out[n] = L->rec[n];
  return 0;
}

/* ComputeMomentumExchangeBodyForce, Source/IBM/IBForceEval.cpp:28-191 */
int orc_momentum_exchange(void *h, double x0, double y0, double z0, double R, int one_sided,
                          double *out3) {
  orc_level *L = (orc_level *)h;
  const int Q = L->Q;
  int opp[ILBM_MAX_Q];
  for (int q = 0; q < Q; ++q) {
    opp[q] = -1;
    for (int p = 0; p < Q; ++p)
      if (fabs(L->cx[p] + L->cx[q]) < 1.e-12 && fabs(L->cy[p] + L->cy[q]) < 1.e-12 &&
          fabs(L->cz[p] + L->cz[q]) < 1.e-12) { opp[q] = p; break; }
  }
  double fxf = 0.0, fyf = 0.0, fzf = 0.0;
  const long s = L->gcells;
  const int vk1 = (L->dim == 3) ? L->n[2] : 1;
#define SDIST(X, Y, Z) ((L->dim == 3) ? sqrt(((X) - x0) * ((X) - x0) + ((Y) - y0) * ((Y) - y0) + ((Z) - z0) * ((Z) - z0)) - R \
                                      : sqrt(((X) - x0) * ((X) - x0) + ((Y) - y0) * ((Y) - y0)) - R)
  for (int k = 0; k < vk1; ++k)
    for (int j = 0; j < L->n[1]; ++j)
      for (int i = 0; i < L->n[0]; ++i) {
        const double xc = L->plo[0] + ((double)i + 0.5) * L->dx[0];
        const double yc = L->plo[1] + ((double)j + 0.5) * L->dx[1];
        const double zc = (L->dim == 3) ? L->plo[2] + ((double)k + 0.5) * L->dx[2] : 0.0;
        if (!(SDIST(xc, yc, zc) > 0.0)) continue;
        for (int q = 0; q < Q; ++q) {
          if (fabs(L->cx[q]) < 1.e-12 && fabs(L->cy[q]) < 1.e-12 && fabs(L->cz[q]) < 1.e-12) continue;
          if (opp[q] < 0) continue;
          int in = i + (int)llround(L->cx[q]), jn = j + (int)llround(L->cy[q]);
          int kn = k + (int)llround(L->cz[q]);
          if (L->periodic[0]) { while (in < 0) in += L->n[0]; while (in > L->n[0] - 1) in -= L->n[0]; }
          else if (in < 0 || in > L->n[0] - 1) continue;
          if (L->periodic[1]) { while (jn < 0) jn += L->n[1]; while (jn > L->n[1] - 1) jn -= L->n[1]; }
          else if (jn < 0 || jn > L->n[1] - 1) continue;
          if (L->dim == 3) {
            if (L->periodic[2]) { while (kn < 0) kn += L->n[2]; while (kn > L->n[2] - 1) kn -= L->n[2]; }
            else if (kn < 0 || kn > L->n[2] - 1) continue;
          } else {
            kn = 0;
          }
          const double xn = L->plo[0] + ((double)in + 0.5) * L->dx[0];
          const double yn = L->plo[1] + ((double)jn + 0.5) * L->dx[1];
          const double zn = (L->dim == 3) ? L->plo[2] + ((double)kn + 0.5) * L->dx[2] : 0.0;
          if (!(SDIST(xn, yn, zn) <= 0.0)) continue;
          const double f_out = L->f_new[IX(L, i, j, k) + q * s];
          double dm;
          if (one_sided) dm = 2.0 * f_out;
          else dm = f_out + L->f_new[IX(L, in, jn, kn) + opp[q] * s];
          fxf += dm * L->cx[q];
          fyf += dm * L->cy[q];
          fzf += dm * L->cz[q];
        }
      }
#undef SDIST
  out3[0] = -fxf;
  out3[1] = -fyf;
  out3[2] = -fzf;
  return 0;
}

/* per-cell entry points for unit parity */
double orc_delta_function(double xf, double xp, double h, int type) { return orc_delta(xf, xp, h, type); }
double orc_overlap(double xa, double xb, double h, int type, double plo, int ilo, int ihi) {
  return orc_overlap_1d(xa, xb, h, type, plo, ilo, ihi);
}

/* ------------------------------------------------------------------------ */
/* static hierarchy: AmrCoreLBM::timeStepWithSubcycling                     */
/* (Source/Core/AmrCoreLBM.cpp:1690-1755) for a coarse level equal to the   */
/* domain and one box per finer level (ratio 2, properly nested), fixed (no */
/* regrid)                                                                  */
/* ------------------------------------------------------------------------ */
#define ORC_MAX_LEV 8
typedef struct {
  int n;
  orc_level *lv[ORC_MAX_LEV];
  int lo[ORC_MAX_LEV][3], hi[ORC_MAX_LEV][3]; /* level boxes in their own domain indices */
} orc_hier;

/* amrex::average_down of ratio 2 (AverageDownTo, AmrCoreLBM.cpp:1519-1527):
 * each coarse cell covered by the fine box [flo, fhi] gets the mean of its
 * fine cells, summed k, j, i inner and scaled by the volume fraction */
static void average_down(const orc_level *C, const orc_level *F, const int *flo, const int *fhi,
                         const double *fine, double *crse, int nc) {
  const int kr = (C->dim == 3) ? 2 : 1;
  const double volfrac = (C->dim == 3) ? 0.125 : 0.25;
  const int ck0 = (C->dim == 3) ? flo[2] / 2 : 0, ck1 = (C->dim == 3) ? fhi[2] / 2 : 0;
  const int cz = (C->dim == 3) ? C->cflo[2] : 0;
  for (int n = 0; n < nc; ++n)
    for (int kc = ck0; kc <= ck1; ++kc)
      for (int jc = flo[1] / 2; jc <= fhi[1] / 2; ++jc)
        for (int ic = flo[0] / 2; ic <= fhi[0] / 2; ++ic) {
          double c = 0.0;
          for (int kk = 0; kk < kr; ++kk)
            for (int jj = 0; jj < 2; ++jj)
              for (int ii = 0; ii < 2; ++ii) {
                const int fi = 2 * ic + ii - flo[0], fj = 2 * jc + jj - flo[1];
                const int fk = (C->dim == 3) ? 2 * kc + kk - flo[2] : 0;
                c += fine[IX(F, fi, fj, fk) + (long)n * F->gcells];
              }
          crse[IX(C, ic - C->cflo[0], jc - C->cflo[1], kc - cz) + (long)n * C->gcells] = volfrac * c;
        }
}

/* coarse case c and nlev - 1 finer boxes: box l (l = 1..nlev-1) is
 * lohi[6(l-1) .. 6(l-1)+5] = lo xyz, hi xyz in level l's domain indices (even
 * lo, odd hi, its coarsened box at least two cells inside level l-1's box,
 * and inside the domain by two cells for level 1) */
void *orcN_create(const ilbm_case *c, int nlev, const int *lohi) {
  if (nlev < 1 || nlev > ORC_MAX_LEV) return NULL;
  orc_hier *H = (orc_hier *)calloc(1, sizeof(orc_hier));
  H->n = nlev;
  for (int d = 0; d < 3; ++d) {
    H->lo[0][d] = 0;
    H->hi[0][d] = (d < c->dim) ? c->n_cell[d] - 1 : 0;
  }
  for (int l = 1; l < nlev; ++l)
    for (int d = 0; d < 3; ++d) {
      H->lo[l][d] = (d < c->dim) ? lohi[6 * (l - 1) + d] : 0;
      H->hi[l][d] = (d < c->dim) ? lohi[6 * (l - 1) + 3 + d] : 0;
      if (d >= c->dim) continue;
      const int plo = H->lo[l - 1][d], phi = H->hi[l - 1][d];
      if ((H->lo[l][d] & 1) || !(H->hi[l][d] & 1) || H->hi[l][d] < H->lo[l][d] ||
          H->lo[l][d] / 2 < plo + 2 || H->hi[l][d] / 2 > phi - 2) {
        free(H);
        return NULL;
      }
    }
  H->lv[0] = (orc_level *)orc_create(c);
  if (!H->lv[0]) { free(H); return NULL; }
  double dx = (c->prob_hi[0] - c->prob_lo[0]) / (double)c->n_cell[0];
  for (int l = 1; l < nlev; ++l) {
    dx *= 0.5;
    ilbm_case fc = *c;
    for (int d = 0; d < 3; ++d) {
      if (d < c->dim) {
        fc.n_cell[d] = H->hi[l][d] - H->lo[l][d] + 1;
        fc.prob_lo[d] = c->prob_lo[d] + dx * (double)H->lo[l][d];
        fc.prob_hi[d] = c->prob_lo[d] + dx * (double)(H->hi[l][d] + 1);
      }
      fc.periodic[d] = 0;
      fc.bc_lo[d] = fc.bc_hi[d] = BC_FOEXTRAP; /* unused: every ghost is coarse-fine */
    }
    H->lv[l] = (orc_level *)orc_create(&fc);
    if (!H->lv[l]) return NULL;
    H->lv[l]->cf = H->lv[l - 1];
    for (int d = 0; d < 3; ++d) H->lv[l]->cflo[d] = H->lo[l][d];
  }
  return H;
}

void orcN_destroy(void *h) {
  orc_hier *H = (orc_hier *)h;
  for (int l = 0; l < H->n; ++l) orc_destroy(H->lv[l]);
  free(H);
}

void *orcN_level(void *h, int lev) { return ((orc_hier *)h)->lv[lev]; }

/* timeStepWithSubcycling(lev): the level's step from its current time, then
 * (below the finest level) two substeps of the next finer level with their
 * coarse-fine ghosts at t and t + dt/2, then the average-down onto it */
static void orcN_advance(orc_hier *H, int lev) {
  orc_level *L = H->lv[lev];
  const double t_old = L->time, t_new = L->time + L->dt;
  level_step(L);
  L->time = t_new;
  L->step += 1;
  if (lev + 1 >= H->n) return;
  orc_level *F = H->lv[lev + 1];
  for (int sub = 0; sub < 2; ++sub) {
    const double t = t_old + (double)sub * F->dt;
    /* GetDataMacro(lev, t): within teps of t_new / t_old, else both */
    const double teps = dmax(1.e-12, fabs(t_new - t_old) * 1.e-3);
    if (t >= t_new - teps && t <= t_new + teps) F->cf_mode = 1;
    else if (t >= t_old - teps && t <= t_old + teps) F->cf_mode = 0;
    else {
      F->cf_mode = 2;
      F->cf_a = (t_new - t) / (t_new - t_old);
      F->cf_b = (t - t_old) / (t_new - t_old);
    }
    F->time = t;
    orcN_advance(H, lev + 1);
  }
  F->time = t_new;
  average_down(L, F, H->lo[lev + 1], H->hi[lev + 1], F->f_new, L->f_new, L->Q);
  average_down(L, F, H->lo[lev + 1], H->hi[lev + 1], F->mac_new, L->mac_new, 6);
}

/* coarse steps of the whole hierarchy; the force record of the finest level
 * once per coarse step (Evolve, AmrCoreLBM.cpp:361-420) */
int orcN_step(void *h, int nsteps) {
  orc_hier *H = (orc_hier *)h;
  for (int s = 0; s < nsteps; ++s) {
    orcN_advance(H, 0);
    compute_ib_force(H->lv[H->n - 1]);
  }
  return 0;
}

/* InitData (AmrCoreLBM.cpp:704-722): each level's equilibrium from its own
 * macro fields, then AverageDown from the finest level to the coarsest and
 * macro_old = macro_new on the levels that have a finer one */
int orcN_init_equilibrium(void *h) {
  orc_hier *H = (orc_hier *)h;
  for (int l = 0; l < H->n; ++l) orc_init_equilibrium(H->lv[l]);
  for (int l = H->n - 1; l > 0; --l) {
    orc_level *C = H->lv[l - 1], *F = H->lv[l];
    average_down(C, F, H->lo[l], H->hi[l], F->f_new, C->f_new, C->Q);
    average_down(C, F, H->lo[l], H->hi[l], F->mac_new, C->mac_new, 6);
  }
  for (int l = 0; l + 1 < H->n; ++l) {
    orc_level *C = H->lv[l];
    memcpy(C->mac_old, C->mac_new, sizeof(double) * 6 * C->gcells);
    memcpy(C->f_old, C->f_new, sizeof(double) * C->Q * C->gcells);
  }
  return 0;
}

/* the two-level hierarchy of the same driver: coarse case c, fine box
 * [flo, fhi] (fine-domain indices) */
void *orc2_create(const ilbm_case *c, const int *flo, const int *fhi) {
  int lohi[6];
  for (int d = 0; d < 3; ++d) {
    lohi[d] = (d < c->dim) ? flo[d] : 0;
    lohi[3 + d] = (d < c->dim) ? fhi[d] : 0;
  }
  return orcN_create(c, 2, lohi);
}
void orc2_destroy(void *h) { orcN_destroy(h); }
void *orc2_level(void *h, int lev) { return orcN_level(h, lev); }
int orc2_step(void *h, int nsteps) { return orcN_step(h, nsteps); }
int orc2_init_equilibrium(void *h) { return orcN_init_equilibrium(h); }
