// Static two-level hierarchy: a coarse level equal to the domain and one
// fine box of refinement ratio 2 inside it, advanced the way
// AmrCoreLBM::timeStepWithSubcycling does (Source/Core/AmrCoreLBM.cpp:
// 1690-1755): one coarse step, two fine substeps, average-down.
//
//   k_cf_fill<L,S>    the fine level's ghost cells for one substep: the
//                     coarse macro fields at the substep's time (old, new or
//                     their linear time interpolation, GetDataMacro
//                     :2239-2269), interpolated to the fine ghost cell by
//                     cell-conservative linear interpolation with
//                     monotonised-central limited slopes (AMReX's
//                     cell_cons_interp, FillPatchMacro :2166-2198); the ghost
//                     populations are the equilibrium of that macro state
//                     (FillPatchMesoscopic's coarse-fine overwrite,
//                     :1566-1626).  One thread per cell of the ghost shell.
//   k_avg_down<L,S>   amrex::average_down of ratio 2 (AverageDownTo,
//                     :1519-1527) of the fine populations and macro fields
//                     onto the covered coarse cells, one thread per coarse
//                     cell: the sum of the 2^d fine cells (k, j, i inner)
//                     times the volume fraction.  The fine macro fields are
//                     those of the fine populations with the last substep's
//                     force (calculateMacroForcing), computed from the
//                     populations the kernel loads anyway.
// Both are HBM-bound gathers; FP64 storage reproduces the oracle's
// arithmetic bit for bit (separately rounded products and sums).

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "batch_internal.h"
#include "ilbm_b200.h"
#include "ilbm_common.cuh"

namespace ilbm {
namespace {

struct CFArgs {
  int lo[3], hi[3];        // fine box, fine-domain indices
  int gf, gm;              // ghost widths of the fine f / macro arrays
  int64_t fs0, fs1, fs2;   // fine f strides
  int64_t ms0, ms1, ms2;   // fine macro strides
  void *f;                 // fine f_in (storage type)
  void *m;                 // fine macro_in (real type, rho u v w) or NULL
  const void *cold, *cnew; // coarse macro at the coarse step's start / end
  int clo[3], cgm;         // coarse box lo and macro ghost width
  int64_t cs0, cs1, cs2;   // coarse macro strides
  int mode;                // 0 old, 1 new, 2 a * old + b * new
  double a, b;
  float f16_scale;
};

template <class L, class R>
__device__ __forceinline__ double coarse_at(const CFArgs &g, int n, int i, int j, int k) {
  const int64_t e = (int64_t)(i - g.clo[0] + g.cgm) + (int64_t)(j - g.clo[1] + g.cgm) * g.cs0 +
                    ((L::D == 3) ? (int64_t)(k - g.clo[2] + g.cgm) * g.cs1 : 0) + (int64_t)n * g.cs2;
  const R *o = static_cast<const R *>(g.cold), *w = static_cast<const R *>(g.cnew);
  if (g.mode == 0) return double(o[e]);
  if (g.mode == 1) return double(w[e]);
  return X::add(X::mul(g.a, double(o[e])), X::mul(g.b, double(w[e])));
}

__device__ __forceinline__ double mc_slope(double cl, double c, double cr) {
  const double dc = X::mul(0.5, X::sub(cr, cl)), dl = X::sub(c, cl), dr = X::sub(cr, c);
  if (X::mul(dl, dr) <= 0.0) return 0.0;
  double m = fabs(dc);
  m = fmin(m, X::mul(2.0, fabs(dl)));
  m = fmin(m, X::mul(2.0, fabs(dr)));
  return (dc < 0.0) ? -m : m;
}

__device__ __forceinline__ int floor_half(int v) { return (v >= 0) ? v / 2 : -((1 - v) / 2); }

// The ghost shell of width w around the fine box, as one slab per
// dimension: slab d holds the cells outside the box in dimension d and inside
// it in every dimension below d (grown range in the dimensions above), so
// every shell cell is counted once.
template <int D>
struct Shell {
  int lo[3], n[3], w;  // box lo, box extents, shell width
  int64_t off[4];      // first shell index of each slab, and the total
  __host__ __device__ void init(const int *blo, const int *bhi, int width) {
    w = width;
    for (int d = 0; d < 3; ++d) {
      lo[d] = blo[d];
      n[d] = (d < D) ? bhi[d] - blo[d] + 1 : 1;
    }
    off[0] = 0;
    for (int d = 0; d < 3; ++d) {
      int64_t c = 0;
      if (d < D) {
        c = 2 * w;
        for (int e = 0; e < D; ++e)
          if (e != d) c *= (e < d) ? n[e] : n[e] + 2 * w;
      }
      off[d + 1] = off[d] + c;
    }
  }
  __host__ __device__ int64_t total() const { return off[3]; }
  // cell t of the shell (fine-domain indices)
  __device__ void cell(int64_t t, int *g) const {
    const int d = (t >= off[1]) + (t >= off[2]);
    int64_t r = t - (d == 0 ? off[0] : (d == 1 ? off[1] : off[2]));
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      if (e >= D) {
        g[e] = 0;
        continue;
      }
      const int ext = (e == d) ? 2 * w : ((e < d) ? n[e] : n[e] + 2 * w);
      const int c = (int)(r % ext);
      r /= ext;
      if (e == d) g[e] = (c < w) ? lo[e] - w + c : lo[e] + n[e] + (c - w);
      else if (e < d) g[e] = lo[e] + c;
      else g[e] = lo[e] - w + c;
    }
  }
};

template <class L, int S>
__global__ void __launch_bounds__(256) k_cf_fill(CFArgs g, Shell<L::D> sh) {
  using T = typename Store<S>::T;
  using R = typename Store<S>::R;
  const int64_t n = sh.total();
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    int fi[3];
    sh.cell(t, fi);
    int layer = 0;  // Chebyshev distance outside the box
#pragma unroll
    for (int d = 0; d < L::D; ++d)
      layer = max(layer, max(g.lo[d] - fi[d], fi[d] - g.hi[d]));
    int ic[3] = {0, 0, 0};
    double off[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int d = 0; d < L::D; ++d) {
      ic[d] = floor_half(fi[d]);
      off[d] = (fi[d] - 2 * ic[d] == 0) ? -0.25 : 0.25;
    }
    double mv[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if (L::D == 2 && c == 3) {
        mv[c] = 0.0;
        continue;
      }
      const double cc = coarse_at<L, R>(g, c, ic[0], ic[1], ic[2]);
      double v = cc;
#pragma unroll
      for (int d = 0; d < L::D; ++d) {
        int lo3[3] = {ic[0], ic[1], ic[2]}, hi3[3] = {ic[0], ic[1], ic[2]};
        lo3[d] -= 1;
        hi3[d] += 1;
        const double cl = coarse_at<L, R>(g, c, lo3[0], lo3[1], lo3[2]);
        const double cr = coarse_at<L, R>(g, c, hi3[0], hi3[1], hi3[2]);
        v = X::add(v, X::mul(mc_slope(cl, cc, cr), off[d]));
      }
      mv[c] = v;
    }
    if (g.m) {
      const int64_t mi = (int64_t)(fi[0] - g.lo[0] + g.gm) + (int64_t)(fi[1] - g.lo[1] + g.gm) * g.ms0 +
                         ((L::D == 3) ? (int64_t)(fi[2] - g.lo[2] + g.gm) * g.ms1 : 0);
      R *m = static_cast<R *>(g.m);
#pragma unroll
      for (int c = 0; c < 4; ++c) m[mi + c * g.ms2] = R(mv[c]);
    }
    if (layer > g.gf) continue;
    const int64_t bi = (int64_t)(fi[0] - g.lo[0] + g.gf) + (int64_t)(fi[1] - g.lo[1] + g.gf) * g.fs0 +
                       ((L::D == 3) ? (int64_t)(fi[2] - g.lo[2] + g.gf) * g.fs1 : 0);
    T *f = static_cast<T *>(g.f);
    if (S == ILBM_STORAGE_F64) {
      const double r = fmax(mv[0], 1.e-12);
#pragma unroll
      for (int q = 0; q < L::Q; ++q)
        reinterpret_cast<double *>(f)[bi + q * g.fs2] = feq64_3<L>(q, r, mv[1], mv[2], mv[3]);
    } else {
      const float r = fmaxf(float(mv[0]), 1.e-12f);
      const float u = float(mv[1]), v = float(mv[2]), w = float(mv[3]);
#pragma unroll
      for (int q = 0; q < L::Q; ++q) {
        const float s = (S == ILBM_STORAGE_F16_SCALED) ? float(L::w(q)) / g.f16_scale : 1.0f;
        Store<S>::store(f + bi + q * g.fs2, feqs<L>(q, r - 1.0f, u, v, w), s);
      }
    }
  }
}

struct AvgArgs {
  int clo_box[3];          // covered coarse cells: [clo_box, chi_box]
  int chi_box[3];
  int flo[3];              // fine box lo (fine-domain indices)
  int fgf, fgm, cgf, cgm;  // ghost widths
  int64_t ffs0, ffs1, ffs2, fms0, fms1, fms2;  // fine strides (f, macro)
  int64_t cfs0, cfs1, cfs2, cms0, cms1, cms2;  // coarse strides
  int cblo[3];             // coarse box lo
  const void *ff, *fm;     // fine f, fine stored macro (NULL: from f and F)
  void *cf, *cm;           // coarse f, macro
  const void *fF;          // fine force of the last substep (NULL: uniform or zero)
  int rlo[3], rhi[3];      // the fine force array's region (zero outside)
  int use_uniform;
  double uf[3];
  float f16_scale;
};

// rho, u, v, w of a fine cell from its populations (already loaded) and the
// force of the substep that produced them (calculateMacroForcing), or its
// stored value
template <class L, int S>
__device__ __forceinline__ void fine_macro(const AvgArgs &g, const typename Store<S>::R *f, int64_t fmi,
                                           int fi, int fj, int fk, double *m4) {
  using R = typename Store<S>::R;
  if (g.fm) {
    const R *fm = static_cast<const R *>(g.fm);
#pragma unroll
    for (int c = 0; c < 4; ++c) m4[c] = (L::D == 2 && c == 3) ? 0.0 : double(fm[fmi + c * g.fms2]);
    return;
  }
  const int gi[3] = {fi + g.flo[0], fj + g.flo[1], fk + g.flo[2]};
  double F3[3] = {0.0, 0.0, 0.0};
  if (g.fF) {
    bool in = true;
#pragma unroll
    for (int d = 0; d < L::D; ++d) in = in && gi[d] >= g.rlo[d] && gi[d] <= g.rhi[d];
    if (in) {
      const R *F = static_cast<const R *>(g.fF);
      F3[0] = double(F[fmi]);
      F3[1] = double(F[fmi + g.fms2]);
      F3[2] = (L::D == 3) ? double(F[fmi + 2 * g.fms2]) : 0.0;
    }
  } else if (g.use_uniform) {
    F3[0] = g.uf[0];
    F3[1] = g.uf[1];
    F3[2] = (L::D == 3) ? g.uf[2] : 0.0;
  }
  if (S == ILBM_STORAGE_F64) {
    moments64<L>(reinterpret_cast<const double *>(f), F3[0], F3[1], F3[2], m4[0], m4[1], m4[2], m4[3]);
    if (L::D != 3) m4[3] = 0.0;
  } else {
    float dr, u, v, w;
    moments32<L>(reinterpret_cast<const float *>(f), float(F3[0]), float(F3[1]), float(F3[2]), dr, u,
                 v, w);
    m4[0] = 1.0 + double(dr);
    m4[1] = u;
    m4[2] = v;
    m4[3] = (L::D == 3) ? double(w) : 0.0;
  }
}

// one coarse cell per thread, its 2^d fine cells visited once each (k, j, i
// inner): populations summed per direction, macro fields summed, both scaled
// by the volume fraction
template <class L, int S>
__global__ void __launch_bounds__(256) k_avg_down(AvgArgs g) {
  using T = typename Store<S>::T;
  using R = typename Store<S>::R;
  const int nx = g.chi_box[0] - g.clo_box[0] + 1, ny = g.chi_box[1] - g.clo_box[1] + 1;
  const int nz = (L::D == 3) ? g.chi_box[2] - g.clo_box[2] + 1 : 1;
  const int64_t n = (int64_t)nx * ny * nz;
  constexpr int kr = (L::D == 3) ? 2 : 1;
  const T *ff = static_cast<const T *>(g.ff);
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int ic = g.clo_box[0] + (int)(t % nx), jc = g.clo_box[1] + (int)((t / nx) % ny);
    const int kc = (L::D == 3) ? g.clo_box[2] + (int)(t / ((int64_t)nx * ny)) : 0;
    R acc[L::Q];
#pragma unroll
    for (int q = 0; q < L::Q; ++q) acc[q] = R(0);
    double accm[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int kk = 0; kk < kr; ++kk)
#pragma unroll
      for (int jj = 0; jj < 2; ++jj)
#pragma unroll
        for (int ii = 0; ii < 2; ++ii) {
          const int fi = 2 * ic + ii - g.flo[0], fj = 2 * jc + jj - g.flo[1];
          const int fk = (L::D == 3) ? 2 * kc + kk - g.flo[2] : 0;
          const int64_t fb = (int64_t)(fi + g.fgf) + (int64_t)(fj + g.fgf) * g.ffs0 +
                             ((L::D == 3) ? (int64_t)(fk + g.fgf) * g.ffs1 : 0);
          const int64_t fmi = (int64_t)(fi + g.fgm) + (int64_t)(fj + g.fgm) * g.fms0 +
                              ((L::D == 3) ? (int64_t)(fk + g.fgm) * g.fms1 : 0);
          R f[L::Q];
#pragma unroll
          for (int q = 0; q < L::Q; ++q) {
            const float sc = (S == ILBM_STORAGE_F16_SCALED) ? float(L::w(q)) / g.f16_scale : 1.0f;
            f[q] = Store<S>::cvt(ff[fb + q * g.ffs2], sc);
          }
#pragma unroll
          for (int q = 0; q < L::Q; ++q) {
            if (S == ILBM_STORAGE_F64)
              acc[q] = R(X::add(double(acc[q]), double(f[q])));
            else
              acc[q] += f[q];
          }
          double m4[4];
          fine_macro<L, S>(g, f, fmi, fi, fj, fk, m4);
#pragma unroll
          for (int c = 0; c < 4; ++c) accm[c] = X::add(accm[c], m4[c]);
        }
    const int64_t cb = (int64_t)(ic - g.cblo[0] + g.cgf) + (int64_t)(jc - g.cblo[1] + g.cgf) * g.cfs0 +
                       ((L::D == 3) ? (int64_t)(kc - g.cblo[2] + g.cgf) * g.cfs1 : 0);
    const int64_t cmi = (int64_t)(ic - g.cblo[0] + g.cgm) + (int64_t)(jc - g.cblo[1] + g.cgm) * g.cms0 +
                        ((L::D == 3) ? (int64_t)(kc - g.cblo[2] + g.cgm) * g.cms1 : 0);
    T *cf = static_cast<T *>(g.cf);
#pragma unroll
    for (int q = 0; q < L::Q; ++q) {
      const float sc = (S == ILBM_STORAGE_F16_SCALED) ? float(L::w(q)) / g.f16_scale : 1.0f;
      if (S == ILBM_STORAGE_F64)
        reinterpret_cast<double *>(cf)[cb + q * g.cfs2] = X::mul((L::D == 3) ? 0.125 : 0.25, double(acc[q]));
      else
        Store<S>::store(cf + cb + q * g.cfs2, ((L::D == 3) ? 0.125f : 0.25f) * float(acc[q]), sc);
    }
    R *cm = static_cast<R *>(g.cm);
    const int ncm = (L::D == 3) ? 4 : 3;
    for (int c4 = 0; c4 < ncm; ++c4) cm[cmi + c4 * g.cms2] = R(X::mul((L::D == 3) ? 0.125 : 0.25, accm[c4]));
  }
}

int grid_of(const ilbm_ctx *ctx, int64_t n) {
  const int64_t cap = (int64_t)std::max(ctx->sms, 1) * 16;
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, cap));
}

template <class L, int S>
int launch_cf_fill(ilbm_ctx *ctx, const CFArgs &g) {
  // macro ghosts (width gm) only when the substep reads stored macro fields
  Shell<L::D> sh;
  sh.init(g.lo, g.hi, g.m ? g.gm : g.gf);
  k_cf_fill<L, S><<<grid_of(ctx, sh.total()), 256, 0, ctx->stream>>>(g, sh);
  ctx->launches++;
  return ILBM_OK;
}

template <class L, int S>
int launch_avg_down(ilbm_ctx *ctx, const AvgArgs &g) {
  int64_t n = 1;
  for (int d = 0; d < L::D; ++d) n *= (int64_t)(g.chi_box[d] - g.clo_box[d] + 1);
  k_avg_down<L, S><<<grid_of(ctx, n), 256, 0, ctx->stream>>>(g);
  ctx->launches++;
  return ILBM_OK;
}

double f16_scale_of(const ilbm_level_params *p) {
  return (p && p->f16_scale > 0.0) ? p->f16_scale : 1024.0;
}

// the hierarchy's shape: fine box aligned to coarse cells and two coarse
// cells inside the domain, fine domain twice the coarse one, ghost modes
int check_two_level(const ilbm_ctx *ctx, const ilbm_box *c, const ilbm_level_params *pc,
                    const ilbm_box *f, const ilbm_level_params *pf) {
  auto fail = [](const char *m) {
    set_error(std::string("two-level hierarchy: ") + m);
    return ILBM_ERR_ARG;
  };
  if (pc->ghost_mode != ILBM_GHOST_SELF) return fail("the coarse level self-fills its ghosts");
  if (pf->ghost_mode != ILBM_GHOST_CALLER) return fail("the fine level takes its ghosts from the coarse level (ILBM_GHOST_CALLER)");
  if (pf->nlevel_boxes > 1) return fail("one fine box");
  for (int d = 0; d < ctx->dim; ++d) {
    if (c->lo[d] != pc->domain_lo[d] || c->hi[d] != pc->domain_hi[d]) return fail("the coarse box must equal its domain");
    if (pf->domain_lo[d] != 2 * pc->domain_lo[d] || pf->domain_hi[d] != 2 * pc->domain_hi[d] + 1)
      return fail("the fine domain must be the coarse domain refined by 2");
    if ((f->lo[d] & 1) || !(f->hi[d] & 1) || f->hi[d] < f->lo[d]) return fail("the fine box must cover whole coarse cells");
    if (f->lo[d] / 2 < pc->domain_lo[d] + 2 || f->hi[d] / 2 > pc->domain_hi[d] - 2)
      return fail("the fine box must lie two coarse cells inside the domain");
  }
  if (f->ngrow_f < 1 || f->ngrow_m < 1 || c->ngrow_m < 1) return fail("ghost widths must be at least 1");
  if (!c->macro_in || !c->macro_out)
    return fail("the coarse level carries stored macro fields (macro_in and macro_out)");
  return ILBM_OK;
}

AvgArgs avg_args(const ilbm_ctx *ctx, const ilbm_box *c, const ilbm_box *f, const void *ff,
                 const void *fm, void *cf, void *cm, const ilbm_level_params *p) {
  AvgArgs g;
  std::memset(&g, 0, sizeof(g));
  for (int d = 0; d < 3; ++d) {
    const bool use = d < ctx->dim;
    g.clo_box[d] = use ? f->lo[d] / 2 : 0;
    g.chi_box[d] = use ? f->hi[d] / 2 : 0;
    g.flo[d] = use ? f->lo[d] : 0;
    g.cblo[d] = use ? c->lo[d] : 0;
  }
  g.fgf = f->ngrow_f;
  g.fgm = f->ngrow_m;
  g.cgf = c->ngrow_f;
  g.cgm = c->ngrow_m;
  g.ffs0 = f->fstride[0]; g.ffs1 = f->fstride[1]; g.ffs2 = f->fstride[2];
  g.fms0 = f->mstride[0]; g.fms1 = f->mstride[1]; g.fms2 = f->mstride[2];
  g.cfs0 = c->fstride[0]; g.cfs1 = c->fstride[1]; g.cfs2 = c->fstride[2];
  g.cms0 = c->mstride[0]; g.cms1 = c->mstride[1]; g.cms2 = c->mstride[2];
  g.ff = ff;
  g.fm = fm;
  g.cf = cf;
  g.cm = cm;
  g.f16_scale = (float)f16_scale_of(p);
  if (p->use_uniform_force) {
    g.use_uniform = 1;
    for (int d = 0; d < 3; ++d) g.uf[d] = p->uniform_force[d];
  }
  return g;
}

}  // namespace
}  // namespace ilbm

using namespace ilbm;

extern "C" {

int ilbm_average_down(ilbm_ctx *ctx, const ilbm_box *coarse, const ilbm_level_params *pc,
                      const ilbm_box *fine, const ilbm_level_params *pf) {
  if (!ctx || !coarse || !pc || !fine || !pf || !coarse->f_in || !fine->f_in || !coarse->macro_in ||
      !fine->macro_in) {
    set_error("ilbm_average_down: null argument");
    return ILBM_ERR_ARG;
  }
  ilbm_box c = *coarse, f = *fine;
  c.macro_out = c.macro_in;
  // any pair of adjacent levels of a hierarchy: the coarser one equal to its
  // domain (self-filled) or one box of a level in between
  int rc;
  if (pc->ghost_mode == ILBM_GHOST_SELF) {
    if ((rc = check_two_level(ctx, &c, pc, &f, pf))) return rc;
  } else {
    for (int d = 0; d < ctx->dim; ++d)
      if ((f.lo[d] & 1) || !(f.hi[d] & 1) || f.lo[d] / 2 < c.lo[d] + 2 || f.hi[d] / 2 > c.hi[d] - 2 ||
          pf->domain_lo[d] != 2 * pc->domain_lo[d] || pf->domain_hi[d] != 2 * pc->domain_hi[d] + 1) {
        set_error("ilbm_average_down: the fine box must cover whole coarse cells two cells inside the "
                  "coarse box, on the coarse domain refined by 2");
        return ILBM_ERR_ARG;
      }
  }
  const AvgArgs g = avg_args(ctx, &c, &f, f.f_in, f.macro_in, c.f_in, c.macro_in, pf);
  return ILBM_DISPATCH(ctx, launch_avg_down, ctx, g);
}

}  // extern "C"

namespace {

// a force record requested with the step: region [lo, hi] of the fine
// level's force of the second substep, written to rec (device-accessible)
struct StepRecord {
  const int *lo, *hi;
  double *rec;
};

int advance_two_level_impl(ilbm_ctx *ctx, const ilbm_box *coarse, const ilbm_level_params *pc,
                           const ilbm_box *fine, const ilbm_level_params *pf, ilbm_ib *ib,
                           double dt, double time, int flags, const StepRecord *record) {
  if (!ctx || !coarse || !pc || !fine || !pf) {
    set_error("ilbm_advance_two_level: null argument");
    return ILBM_ERR_ARG;
  }
  int rc = check_two_level(ctx, coarse, pc, fine, pf);
  if (rc) return rc;
  if (!coarse->f_out || !fine->f_out) {
    set_error("ilbm_advance_two_level: f_out must be set on both levels");
    return ILBM_ERR_ARG;
  }
  if (ib && (!fine->force || !fine->force_prev)) {
    set_error("ilbm_advance_two_level: a body needs the fine level's force and force_prev");
    return ILBM_ERR_ARG;
  }
  const bool first = (flags & ILBM_TWO_LEVEL_FIRST_STEP) != 0;
  if (first && !fine->macro_in) {
    set_error("ilbm_advance_two_level: the first step reads the fine level's stored macro_in");
    return ILBM_ERR_ARG;
  }
  const double t_old = time, t_new = time + dt, dtf = 0.5 * dt;
  // Schedule.  The first substep reads the coarse data at t_old only, so the
  // coarse step need not precede it; the second substep's ghosts need the
  // coarse step's result.  With a body, each substep's forcing chain runs on
  // the side stream beside work of the main stream: the first substep's
  // beside the first half of the coarse step and the substep's cells outside
  // the body's band, the second substep's (which needs the first substep's
  // band) beside the second half of the coarse step and the second
  // substep's outer cells.
  ilbm_box b0 = *fine;
  b0.macro_in = first ? fine->macro_in : nullptr;
  b0.macro_out = nullptr;
  AdvanceSplit sp0;
  if (ib && (rc = advance_begin(ctx, &b0, pf, ib, dtf, t_old, &sp0))) return rc;
  // coarse step (no body: the body lives on the finest level).  Its stored
  // macro fields are kept on the covered cells grown by two coarse cells --
  // what average-down writes and the fine ghost fill reads; elsewhere they
  // equal the populations' own and are recovered from them
  int mlo[3] = {0, 0, 0}, mhi[3] = {0, 0, 0};
  for (int d = 0; d < ctx->dim; ++d) {
    mlo[d] = fine->lo[d] / 2 - 2;
    mhi[d] = fine->hi[d] / 2 + 2;
  }
  const int *cmlo = first ? nullptr : mlo, *cmhi = first ? nullptr : mhi;
  if ((rc = level_step_impl(ctx, coarse, 1, pc, cmlo, cmhi, ib ? 1 : 0))) return rc;
  CFArgs g;
  std::memset(&g, 0, sizeof(g));
  for (int d = 0; d < 3; ++d) {
    const bool use = d < ctx->dim;
    g.lo[d] = use ? fine->lo[d] : 0;
    g.hi[d] = use ? fine->hi[d] : 0;
    g.clo[d] = use ? coarse->lo[d] : 0;
  }
  g.gf = fine->ngrow_f;
  g.gm = fine->ngrow_m;
  g.fs0 = fine->fstride[0]; g.fs1 = fine->fstride[1]; g.fs2 = fine->fstride[2];
  g.ms0 = fine->mstride[0]; g.ms1 = fine->mstride[1]; g.ms2 = fine->mstride[2];
  g.cgm = coarse->ngrow_m;
  g.cs0 = coarse->mstride[0]; g.cs1 = coarse->mstride[1]; g.cs2 = coarse->mstride[2];
  g.cold = coarse->macro_in;
  g.cnew = coarse->macro_out;
  g.f16_scale = (float)f16_scale_of(pf);
  AdvanceSplit sp1;
  for (int sub = 0; sub < 2; ++sub) {
    // stored fine macro fields only for a first step after initialisation;
    // afterwards rho, u are recovered from f and F^{n-1}
    ilbm_box b = (sub == 0) ? b0 : *fine;
    if (sub == 1) {
      b.macro_in = nullptr;
      b.macro_out = nullptr;
      std::swap(b.f_in, b.f_out);
      std::swap(b.force, b.force_prev);
    }
    const double t = t_old + (double)sub * dtf;
    // GetDataMacro(0, t): the coarse data at t_new, at t_old, or both
    const double teps = std::max(1.e-12, std::fabs(t_new - t_old) * 1.e-3);
    if (t >= t_new - teps && t <= t_new + teps) {
      g.mode = 1;
    } else if (t >= t_old - teps && t <= t_old + teps) {
      g.mode = 0;
    } else {
      g.mode = 2;
      g.a = (t_new - t) / (t_new - t_old);
      g.b = (t - t_old) / (t_new - t_old);
    }
    g.f = b.f_in;
    g.m = b.macro_in;
    if ((rc = ILBM_DISPATCH(ctx, launch_cf_fill, ctx, g))) return rc;
    if (!ib) {
      if ((rc = ilbm_level_step(ctx, &b, 1, pf))) return rc;
    } else if (sub == 0) {
      if ((rc = advance_end(ctx, &b, &sp0))) return rc;
    } else {
      if ((rc = advance_end(ctx, &b, &sp1))) return rc;
    }
    if (ib && sub == 0) {
      // the second substep's forcing (after the first substep's band), then
      // the rest of the coarse step with its stored macro fields, which the
      // second substep's ghost fill reads
      ilbm_box b1 = *fine;
      b1.macro_in = nullptr;
      b1.macro_out = nullptr;
      std::swap(b1.f_in, b1.f_out);
      std::swap(b1.force, b1.force_prev);
      if ((rc = advance_begin(ctx, &b1, pf, ib, dtf, t_old + dtf, &sp1))) return rc;
      // the record reads what the second substep's chain produces (its
      // exported force, the marker force sum, the status): on the side
      // stream right after it, beside the main stream's remaining work,
      // which only reads those arrays
      if (record && !sp1.serial &&
          (rc = ib_record_on(ib, b1, record->lo, record->hi, record->rec, ctx->side)))
        return rc;
      if ((rc = level_step_impl(ctx, coarse, 1, pc, cmlo, cmhi, 2))) return rc;
    }
  }
  // the fine state is back in fine->f_in after two substeps, the force of
  // the second substep in fine->force_prev
  AvgArgs a = avg_args(ctx, coarse, fine, fine->f_in, nullptr, coarse->f_out, coarse->macro_out, pf);
  if (ib) {
    a.fF = fine->force_prev;
    a.use_uniform = 0;
    int lo[3], hi[3];
    ilbm_ib_force_region(ib, lo, hi);
    for (int d = 0; d < 3; ++d) {
      a.rlo[d] = lo[d];
      a.rhi[d] = hi[d];
    }
  }
  if ((rc = ILBM_DISPATCH(ctx, launch_avg_down, ctx, a))) return rc;
  if (record) {
    if (sp1.serial) {  // the chain ran on the main stream: the record follows it there
      ilbm_box rb = *fine;
      rb.force = fine->force_prev;
      if ((rc = ib_record_on(ib, rb, record->lo, record->hi, record->rec, ctx->stream))) return rc;
    }
    // the step's end waits for the record taken beside it
    cudaError_t e = cudaStreamWaitEvent(ctx->stream, ctx->ev_rec, 0);
    if (e != cudaSuccess) return cuda_fail(e, "ilbm_advance_two_level_recorded");
  }
  return ILBM_OK;
}

}  // namespace

extern "C" {

int ilbm_advance_two_level(ilbm_ctx *ctx, const ilbm_box *coarse, const ilbm_level_params *pc,
                           const ilbm_box *fine, const ilbm_level_params *pf, ilbm_ib *ib,
                           double dt, double time, int flags) {
  return advance_two_level_impl(ctx, coarse, pc, fine, pf, ib, dt, time, flags, nullptr);
}

int ilbm_advance_two_level_recorded(ilbm_ctx *ctx, const ilbm_box *coarse,
                                    const ilbm_level_params *pc, const ilbm_box *fine,
                                    const ilbm_level_params *pf, ilbm_ib *ib, double dt,
                                    double time, int flags, const int lo[3], const int hi[3],
                                    double *out) {
  if (!ctx || !ib || !fine || !lo || !hi || !out) {
    set_error("ilbm_advance_two_level_recorded: null argument");
    return ILBM_ERR_ARG;
  }
  // the record's last kernel writes `out` itself when the device can address
  // it (pinned host memory, or memory of this device); other memory gets the
  // step, then the record through ilbm_force_record_async
  double *direct = nullptr;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, out) == cudaSuccess) {
    if (at.type == cudaMemoryTypeHost && at.devicePointer)
      direct = static_cast<double *>(at.devicePointer);
    else if (at.type == cudaMemoryTypeDevice && at.device == ctx->device)
      direct = out;
  }
  cudaGetLastError();  // an unregistered pointer is not an error here
  if (!direct) {
    int rc = advance_two_level_impl(ctx, coarse, pc, fine, pf, ib, dt, time, flags, nullptr);
    if (rc) return rc;
    ilbm_box rb = *fine;
    rb.force = fine->force_prev;
    return ilbm_force_record_async(ctx, &rb, 1, ib, lo, hi, out);
  }
  const StepRecord r{lo, hi, direct};
  return advance_two_level_impl(ctx, coarse, pc, fine, pf, ib, dt, time, flags, &r);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Static hierarchy of any depth: AmrCoreLBM::timeStepWithSubcycling's
// recursion (Source/Core/AmrCoreLBM.cpp:1690-1755).  A level's step, then
// (below the finest level) two substeps of the next finer level, each with
// its ghost cells filled from this level's macro fields at the substep's
// time, then the average-down of that level onto this one (AverageDownTo,
// :1519-1527).  The body, if any, lives on the finest level, whose steps
// overlap the body's forcing chain with the cells outside its band.
// ---------------------------------------------------------------------------
namespace ilbm {
namespace {

struct HLevel {
  ilbm_box b;                     // current buffers (swapped after each step)
  const ilbm_level_params *p;
  bool first;                     // the level's first step reads its stored macro everywhere
  int mlo[3], mhi[3];             // stored macro region: the finer box coarsened, grown by 2
  double t_old, t_new;            // the level's current step
};

int hier_check(const ilbm_ctx *ctx, int nlev, const ilbm_box *boxes, const ilbm_level_params *ps) {
  auto fail = [](const char *m) {
    set_error(std::string("hierarchy: ") + m);
    return ILBM_ERR_ARG;
  };
  if (nlev < 2 || nlev > 8) return fail("2 to 8 levels");
  if (ps[0].ghost_mode != ILBM_GHOST_SELF) return fail("the coarsest level self-fills its ghosts");
  for (int l = 0; l < nlev; ++l) {
    const ilbm_box &b = boxes[l];
    if (!b.f_in || !b.f_out || b.f_in == b.f_out) return fail("every level needs distinct f_in and f_out");
    if (b.ngrow_f < 1 || b.ngrow_m < 1) return fail("ghost widths must be at least 1");
    if (l + 1 < nlev && (!b.macro_in || !b.macro_out))
      return fail("every level with a finer one carries stored macro fields (macro_in and macro_out)");
    if (l == 0) {
      for (int d = 0; d < ctx->dim; ++d)
        if (b.lo[d] != ps[0].domain_lo[d] || b.hi[d] != ps[0].domain_hi[d])
          return fail("the coarsest box must equal its domain");
      continue;
    }
    const ilbm_box &c = boxes[l - 1];
    if (ps[l].ghost_mode != ILBM_GHOST_CALLER)
      return fail("finer levels take their ghosts from the level above (ILBM_GHOST_CALLER)");
    if (ps[l].nlevel_boxes > 1) return fail("one box per level");
    for (int d = 0; d < ctx->dim; ++d) {
      if (ps[l].domain_lo[d] != 2 * ps[l - 1].domain_lo[d] ||
          ps[l].domain_hi[d] != 2 * ps[l - 1].domain_hi[d] + 1)
        return fail("each domain must be the one above refined by 2");
      if ((b.lo[d] & 1) || !(b.hi[d] & 1) || b.hi[d] < b.lo[d])
        return fail("each box must cover whole cells of the level above");
      if (b.lo[d] / 2 < c.lo[d] + 2 || b.hi[d] / 2 > c.hi[d] - 2)
        return fail("each box must lie two cells of the level above inside that level's box");
    }
  }
  return ILBM_OK;
}

// ghost cells of level `lev` for a step at time t, from level lev-1's macro
// fields at its step's start (macro_in) and end (macro_out)
int hier_cf_fill(ilbm_ctx *ctx, const HLevel &C, const HLevel &F, double t, bool reads_macro) {
  CFArgs g;
  std::memset(&g, 0, sizeof(g));
  for (int d = 0; d < 3; ++d) {
    const bool use = d < ctx->dim;
    g.lo[d] = use ? F.b.lo[d] : 0;
    g.hi[d] = use ? F.b.hi[d] : 0;
    g.clo[d] = use ? C.b.lo[d] : 0;
  }
  g.gf = F.b.ngrow_f;
  g.gm = F.b.ngrow_m;
  g.fs0 = F.b.fstride[0]; g.fs1 = F.b.fstride[1]; g.fs2 = F.b.fstride[2];
  g.ms0 = F.b.mstride[0]; g.ms1 = F.b.mstride[1]; g.ms2 = F.b.mstride[2];
  g.cgm = C.b.ngrow_m;
  g.cs0 = C.b.mstride[0]; g.cs1 = C.b.mstride[1]; g.cs2 = C.b.mstride[2];
  g.cold = C.b.macro_in;
  g.cnew = C.b.macro_out;
  g.f16_scale = (float)f16_scale_of(F.p);
  // GetDataMacro(lev-1, t): the data at t_new, at t_old, or both
  const double teps = std::max(1.e-12, std::fabs(C.t_new - C.t_old) * 1.e-3);
  if (t >= C.t_new - teps && t <= C.t_new + teps) {
    g.mode = 1;
  } else if (t >= C.t_old - teps && t <= C.t_old + teps) {
    g.mode = 0;
  } else {
    g.mode = 2;
    g.a = (C.t_new - t) / (C.t_new - C.t_old);
    g.b = (t - C.t_old) / (C.t_new - C.t_old);
  }
  g.f = F.b.f_in;
  g.m = reads_macro ? F.b.macro_in : nullptr;
  return ILBM_DISPATCH(ctx, launch_cf_fill, ctx, g);
}

int hier_advance(ilbm_ctx *ctx, std::vector<HLevel> &H, int lev, ilbm_ib *ib, double dt, double t) {
  const int nlev = (int)H.size();
  const bool finest = lev == nlev - 1;
  HLevel &L = H[lev];
  L.t_old = t;
  L.t_new = t + dt;
  int rc;
  ilbm_box b = L.b;
  if (finest) {
    b.macro_in = L.first ? L.b.macro_in : nullptr;
    b.macro_out = nullptr;
  }
  if (lev > 0 && (rc = hier_cf_fill(ctx, H[lev - 1], L, t, finest && L.first))) return rc;
  if (!finest) {
    // stored macro fields: on the coarsest level on the region the finer
    // level's ghost fill and average-down use (everywhere on its first step);
    // on a level in between everywhere, since the average-down onto the level
    // above takes its stored values (which hold the finer level's average on
    // the covered cells)
    const bool whole = L.first || lev > 0;
    if ((rc = level_step_impl(ctx, &b, 1, L.p, whole ? nullptr : L.mlo, whole ? nullptr : L.mhi, 0)))
      return rc;
  } else if (ib) {
    AdvanceSplit sp;
    if ((rc = advance_begin(ctx, &b, L.p, ib, dt, t, &sp))) return rc;
    if ((rc = advance_end(ctx, &b, &sp))) return rc;
  } else {
    if ((rc = ilbm_level_step(ctx, &b, 1, L.p))) return rc;
  }
  L.first = false;
  if (!finest) {
    const double dtf = 0.5 * dt;
    for (int sub = 0; sub < 2; ++sub)
      if ((rc = hier_advance(ctx, H, lev + 1, ib, dtf, t + (double)sub * dtf))) return rc;
    // the finer level's state is back in its f_in after its two substeps;
    // average it down onto this level's new state
    const HLevel &F = H[lev + 1];
    // a finer level that has a finer one itself passes its stored macro
    // fields (AverageDownTo averages macro_new, which there holds the average
    // of the level below on its covered cells); the finest level's macro
    // fields are those of its populations
    const void *fm = (lev + 1 < nlev - 1) ? F.b.macro_in : nullptr;
    AvgArgs a = avg_args(ctx, &L.b, &F.b, F.b.f_in, fm, L.b.f_out, L.b.macro_out, F.p);
    if (lev + 1 == nlev - 1 && ib) {
      a.fF = F.b.force_prev;  // the force of the finest level's last substep
      a.use_uniform = 0;
      int lo[3], hi[3];
      ilbm_ib_force_region(ib, lo, hi);
      for (int d = 0; d < 3; ++d) {
        a.rlo[d] = lo[d];
        a.rhi[d] = hi[d];
      }
    }
    if ((rc = ILBM_DISPATCH(ctx, launch_avg_down, ctx, a))) return rc;
  }
  // the new state becomes the current one
  std::swap(L.b.f_in, L.b.f_out);
  std::swap(L.b.macro_in, L.b.macro_out);
  if (finest && ib) std::swap(L.b.force, L.b.force_prev);
  return ILBM_OK;
}

}  // namespace
}  // namespace ilbm

extern "C" {

int ilbm_advance_hierarchy(ilbm_ctx *ctx, int nlev, const ilbm_box *boxes,
                           const ilbm_level_params *params, ilbm_ib *ib, double dt, double time,
                           int flags) {
  if (!ctx || !boxes || !params) {
    set_error("ilbm_advance_hierarchy: null argument");
    return ILBM_ERR_ARG;
  }
  int rc = hier_check(ctx, nlev, boxes, params);
  if (rc) return rc;
  const ilbm_box &fb = boxes[nlev - 1];
  if (ib && (!fb.force || !fb.force_prev)) {
    set_error("ilbm_advance_hierarchy: a body needs the finest level's force and force_prev");
    return ILBM_ERR_ARG;
  }
  const bool first = (flags & ILBM_HIERARCHY_FIRST_STEP) != 0;
  if (first && !fb.macro_in) {
    set_error("ilbm_advance_hierarchy: the first step reads the finest level's stored macro_in");
    return ILBM_ERR_ARG;
  }
  std::vector<HLevel> H(nlev);
  for (int l = 0; l < nlev; ++l) {
    H[l].b = boxes[l];
    H[l].p = &params[l];
    H[l].first = first;
    for (int d = 0; d < 3; ++d) {
      const bool use = d < ctx->dim && l + 1 < nlev;
      H[l].mlo[d] = use ? boxes[l + 1].lo[d] / 2 - 2 : 0;
      H[l].mhi[d] = use ? boxes[l + 1].hi[d] / 2 + 2 : 0;
    }
  }
  return hier_advance(ctx, H, 0, ib, dt, time);
}

}  // extern "C"
