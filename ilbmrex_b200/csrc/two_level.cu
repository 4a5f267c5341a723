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
//                     :1566-1626).  One thread per cell of the grown fine box;
//                     valid cells return at once.
//   k_avg_down<L,S>   amrex::average_down of ratio 2 (AverageDownTo,
//                     :1519-1527) of the fine populations and macro fields
//                     onto the covered coarse cells, one thread per coarse
//                     cell: the sum of the 2^d fine cells (k, j, i inner)
//                     times the volume fraction.
// Both are HBM-bound gathers; FP64 storage reproduces the oracle's
// arithmetic bit for bit (separately rounded products and sums).

#include <algorithm>
#include <cmath>
#include <cstring>

#include "ilbm_common.cuh"

namespace ilbm {
namespace {

struct CFArgs {
  int lo[3], hi[3];        // fine box, fine-domain indices
  int gf, gm;              // ghost widths of the fine f / macro arrays
  int64_t fs0, fs1, fs2;   // fine f strides
  int64_t ms0, ms1, ms2;   // fine macro strides
  void *f;                 // fine f_in (storage type)
  void *m;                 // fine macro_in (real type, rho u v w)
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

template <class L, int S>
__global__ void __launch_bounds__(256) k_cf_fill(CFArgs g) {
  using T = typename Store<S>::T;
  using R = typename Store<S>::R;
  const int nx = g.hi[0] - g.lo[0] + 1 + 2 * g.gm, ny = g.hi[1] - g.lo[1] + 1 + 2 * g.gm;
  const int nz = (L::D == 3) ? g.hi[2] - g.lo[2] + 1 + 2 * g.gm : 1;
  const int64_t n = (int64_t)nx * ny * nz;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    int fi[3];
    fi[0] = g.lo[0] - g.gm + (int)(t % nx);
    fi[1] = g.lo[1] - g.gm + (int)((t / nx) % ny);
    fi[2] = (L::D == 3) ? g.lo[2] - g.gm + (int)(t / ((int64_t)nx * ny)) : 0;
    int layer = 0;  // Chebyshev distance outside the box
#pragma unroll
    for (int d = 0; d < L::D; ++d)
      layer = max(layer, max(g.lo[d] - fi[d], fi[d] - g.hi[d]));
    if (layer <= 0) continue;
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
    const int64_t mi = (int64_t)(fi[0] - g.lo[0] + g.gm) + (int64_t)(fi[1] - g.lo[1] + g.gm) * g.ms0 +
                       ((L::D == 3) ? (int64_t)(fi[2] - g.lo[2] + g.gm) * g.ms1 : 0);
    R *m = static_cast<R *>(g.m);
#pragma unroll
    for (int c = 0; c < 4; ++c) m[mi + c * g.ms2] = R(mv[c]);
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
  const void *ff, *fm;     // fine f, macro
  void *cf, *cm;           // coarse f, macro
  float f16_scale;
};

template <class L, int S>
__global__ void __launch_bounds__(256) k_avg_down(AvgArgs g) {
  using T = typename Store<S>::T;
  using R = typename Store<S>::R;
  const int nx = g.chi_box[0] - g.clo_box[0] + 1, ny = g.chi_box[1] - g.clo_box[1] + 1;
  const int nz = (L::D == 3) ? g.chi_box[2] - g.clo_box[2] + 1 : 1;
  const int64_t n = (int64_t)nx * ny * nz;
  const int kr = (L::D == 3) ? 2 : 1;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int ic = g.clo_box[0] + (int)(t % nx), jc = g.clo_box[1] + (int)((t / nx) % ny);
    const int kc = (L::D == 3) ? g.clo_box[2] + (int)(t / ((int64_t)nx * ny)) : 0;
    const int64_t cb = (int64_t)(ic - g.cblo[0] + g.cgf) + (int64_t)(jc - g.cblo[1] + g.cgf) * g.cfs0 +
                       ((L::D == 3) ? (int64_t)(kc - g.cblo[2] + g.cgf) * g.cfs1 : 0);
    const int64_t cmi = (int64_t)(ic - g.cblo[0] + g.cgm) + (int64_t)(jc - g.cblo[1] + g.cgm) * g.cms0 +
                        ((L::D == 3) ? (int64_t)(kc - g.cblo[2] + g.cgm) * g.cms1 : 0);
    int64_t fb[8], fmi[8];
    int nf = 0;
    for (int kk = 0; kk < kr; ++kk)
      for (int jj = 0; jj < 2; ++jj)
        for (int ii = 0; ii < 2; ++ii) {
          const int fi = 2 * ic + ii - g.flo[0], fj = 2 * jc + jj - g.flo[1];
          const int fk = (L::D == 3) ? 2 * kc + kk - g.flo[2] : 0;
          fb[nf] = (int64_t)(fi + g.fgf) + (int64_t)(fj + g.fgf) * g.ffs0 +
                   ((L::D == 3) ? (int64_t)(fk + g.fgf) * g.ffs1 : 0);
          fmi[nf] = (int64_t)(fi + g.fgm) + (int64_t)(fj + g.fgm) * g.fms0 +
                    ((L::D == 3) ? (int64_t)(fk + g.fgm) * g.fms1 : 0);
          ++nf;
        }
    const T *ff = static_cast<const T *>(g.ff);
    T *cf = static_cast<T *>(g.cf);
    if (S == ILBM_STORAGE_F64) {
      const double vf = (L::D == 3) ? 0.125 : 0.25;
      for (int q = 0; q < L::Q; ++q) {
        double c = 0.0;
        for (int e = 0; e < nf; ++e) c = X::add(c, double(ff[fb[e] + q * g.ffs2]));
        reinterpret_cast<double *>(cf)[cb + q * g.cfs2] = X::mul(vf, c);
      }
    } else {
      const float vf = (L::D == 3) ? 0.125f : 0.25f;
      for (int q = 0; q < L::Q; ++q) {
        const float s = (S == ILBM_STORAGE_F16_SCALED) ? float(L::w(q)) / g.f16_scale : 1.0f;
        float c = 0.0f;
        for (int e = 0; e < nf; ++e) c += Store<S>::cvt(ff[fb[e] + q * g.ffs2], s);
        Store<S>::store(cf + cb + q * g.cfs2, vf * c, s);
      }
    }
    const R *fm = static_cast<const R *>(g.fm);
    R *cm = static_cast<R *>(g.cm);
    const int ncm = (L::D == 3) ? 4 : 3;
    for (int c4 = 0; c4 < ncm; ++c4) {
      double c = 0.0;
      for (int e = 0; e < nf; ++e) c = X::add(c, double(fm[fmi[e] + c4 * g.fms2]));
      cm[cmi + c4 * g.cms2] = R(X::mul((L::D == 3) ? 0.125 : 0.25, c));
    }
  }
}

int grid_of(const ilbm_ctx *ctx, int64_t n) {
  const int64_t cap = (int64_t)std::max(ctx->sms, 1) * 16;
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, cap));
}

template <class L, int S>
int launch_cf_fill(ilbm_ctx *ctx, const CFArgs &g) {
  int64_t n = 1;
  for (int d = 0; d < L::D; ++d) n *= (int64_t)(g.hi[d] - g.lo[d] + 1 + 2 * g.gm);
  k_cf_fill<L, S><<<grid_of(ctx, n), 256, 0, ctx->stream>>>(g);
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
  if (!c->macro_in || !c->macro_out || !f->macro_in || !f->macro_out)
    return fail("both levels carry stored macro fields (macro_in and macro_out)");
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
  f.macro_out = f.macro_in;
  int rc = check_two_level(ctx, &c, pc, &f, pf);
  if (rc) return rc;
  const AvgArgs g = avg_args(ctx, &c, &f, f.f_in, f.macro_in, c.f_in, c.macro_in, pf);
  return ILBM_DISPATCH(ctx, launch_avg_down, ctx, g);
}

int ilbm_advance_two_level(ilbm_ctx *ctx, const ilbm_box *coarse, const ilbm_level_params *pc,
                           const ilbm_box *fine, const ilbm_level_params *pf, ilbm_ib *ib,
                           double dt, double time) {
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
  // coarse step (no body: the body lives on the finest level)
  if ((rc = ilbm_advance_level(ctx, coarse, pc, nullptr, dt, time))) return rc;
  const double t_old = time, t_new = time + dt, dtf = 0.5 * dt;
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
  for (int sub = 0; sub < 2; ++sub) {
    ilbm_box b = *fine;
    if (sub == 1) {
      std::swap(b.f_in, b.f_out);
      std::swap(b.macro_in, b.macro_out);
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
    if ((rc = ilbm_advance_level(ctx, &b, pf, ib, dtf, t))) return rc;
  }
  // the fine state is back in fine->f_in / fine->macro_in after two substeps
  const AvgArgs a = avg_args(ctx, coarse, fine, fine->f_in, fine->macro_in, coarse->f_out,
                             coarse->macro_out, pf);
  return ILBM_DISPATCH(ctx, launch_avg_down, ctx, a);
}

}  // extern "C"
