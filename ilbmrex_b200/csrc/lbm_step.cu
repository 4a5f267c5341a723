// Fused collide + stream for one level (the per-level hot path).
//
// Reference semantics (Source/Core/AdvanceLBMAtLevel.cpp:20-386): the level
// step FillPatches f^n into a scratch copy with ghosts, collides the valid
// cells in place (collide_forced with the STORED rho^n, u^n and the new force
// F^n), refreshes periodic / inter-box ghosts with post-collision values,
// writes halfway bounce-back ghosts for user_1 faces, pull-streams into f_new
// and recomputes rho, u with F^n/2.
//
// B200 form: one pass.  Each thread owns one cell y, loads its Q populations
// once (coalesced along i), recovers rho^n and u^n from them (bit-identical to
// the stored macro because the reference computed it from the same f^n and
// F^{n-1}; or reads macro_in), collides, and PUSHES f*(y,q) to f_out(y+c_q,q)
// (wrapping periodic directions).  Populations whose pull source is a ghost
// that nobody pushes from are completed by the thread that owns the
// destination: bounce-back (f*(x,q_bar)), the pre-collision ghost value
// (physical BC / coarse-fine), or, for a ghost covered by another box of the
// level, that ghost collided in place.  Physical ghosts of layer 1 are
// synthesised by a small prepass (self-fill mode) with the reference's
// FillPatch rules, so the main kernel never evaluates boundary formulas.
// Traffic per cell: Q loads + Q stores of the storage type (plus the force
// band); no scratch copies.
#include <algorithm>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ilbm_common.cuh"
#include "step_args.cuh"

namespace ilbm {

static thread_local std::string g_err;
void set_error(const std::string &msg) { g_err = msg; }
const char *get_error() { return g_err.c_str(); }
int cuda_fail(cudaError_t e, const char *what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return ILBM_ERR_CUDA;
}


__device__ __forceinline__ int64_t fidx(const StepArgs &a, int i, int j, int k) {
  return (int64_t)(i - a.fgl[0]) + (int64_t)(j - a.fgl[1]) * a.fs0 +
         (int64_t)(k - a.fgl[2]) * a.fs1;
}
__device__ __forceinline__ int64_t midx(const StepArgs &a, int i, int j, int k) {
  return (int64_t)(i - a.mgl[0]) + (int64_t)(j - a.mgl[1]) * a.ms0 +
         (int64_t)(k - a.mgl[2]) * a.ms1;
}

template <class L>
__device__ __forceinline__ bool in_domain(const StepArgs &a, int i, int j, int k) {
  if (i < a.dlo[0] || i > a.dhi[0] || j < a.dlo[1] || j > a.dhi[1]) return false;
  if (L::D == 3 && (k < a.dlo[2] || k > a.dhi[2])) return false;
  return true;
}

// per-direction storage factor for the F16 form: w_q / scale
template <class L, int S>
__device__ __forceinline__ float sfac(const StepArgs &a, int q) {
  if (S == ILBM_STORAGE_F16_SCALED) return float(L::w(q)) / a.f16_scale;
  return 1.0f;
}

template <class L, int S>
__device__ __forceinline__ typename Store<S>::R ldf(const StepArgs &a, int64_t base, int q) {
  using T = typename Store<S>::T;
  return Store<S>::load(static_cast<const T *>(a.f_in) + base + q * a.fs2, sfac<L, S>(a, q));
}

template <class R>
__device__ __forceinline__ R ldm(const void *p, int64_t idx) {
  return static_cast<const R *>(p)[idx];
}

// force at a cell (F^n or F^{n-1}); zero outside the force region
template <class L, class R>
__device__ __forceinline__ void load_force(const StepArgs &a, const void *F, int i, int j,
                                           int k, R &fx, R &fy, R &fz) {
  if (F == nullptr) {
    if (a.use_uniform) {
      fx = R(a.uf[0]);
      fy = R(a.uf[1]);
      fz = R(a.uf[2]);
    } else {
      fx = fy = fz = R(0);
    }
    return;
  }
  if (i < a.flo[0] || i > a.fhi[0] || j < a.flo[1] || j > a.fhi[1] ||
      (L::D == 3 && (k < a.flo[2] || k > a.fhi[2]))) {
    fx = fy = fz = R(0);
    return;
  }
  const int64_t m = midx(a, i, j, k);
  fx = ldm<R>(F, m);
  fy = ldm<R>(F, m + a.ms2);
  fz = (L::D == 3) ? ldm<R>(F, m + 2 * a.ms2) : R(0);
}

// ---------------------------------------------------------------------------
// Ghost synthesis (pre-collision values of physical-boundary ghosts), with the
// FillPatch semantics the reference relies on: periodic images first, then per
// ghost cell AMReX's foextrap fill followed by mesoscopicBcFill
// (Source/BC/bc_fill.H:303-347: user_2 face mirror > user_1 copy > ext_dir
// non-equilibrium extrapolation, mirror = nearest domain cell).
// ---------------------------------------------------------------------------
template <class L>
__device__ __forceinline__ bool first_face(const StepArgs &a, const int *g, int type, int &bd,
                                           int &lo_side) {
#pragma unroll
  for (int d = 0; d < L::D; ++d) {
    if (g[d] < a.dlo[d] && a.bclo[d] == type) { bd = d; lo_side = 1; return true; }
    if (g[d] > a.dhi[d] && a.bchi[d] == type) { bd = d; lo_side = 0; return true; }
  }
  return false;
}

// Resolve a ghost cell to either a source cell in the domain (copy) or a
// boundary formula on a mirror cell.  kind: 0 copy src, 1 user_1 copy of
// mirror, 2 ext_dir NEQ, 3 user_2 face-mirror NEQ.
template <class L>
__device__ __forceinline__ int ghost_rule(const StepArgs &a, const int *g, int *src, int &bd,
                                          int &lo_side) {
  int cur[3] = {g[0], g[1], g[2]};
  for (int it = 0; it < 4; ++it) {
    bool inside = true, wrappable = true;
#pragma unroll
    for (int d = 0; d < L::D; ++d) {
      const bool out = cur[d] < a.dlo[d] || cur[d] > a.dhi[d];
      if (out) {
        inside = false;
        if (!a.periodic[d]) wrappable = false;
      }
    }
    if (inside || wrappable) {
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        int c = cur[d];
        if (d < L::D && a.periodic[d]) {
          const int n = a.dhi[d] - a.dlo[d] + 1;
          c = a.dlo[d] + (((c - a.dlo[d]) % n) + n) % n;
        }
        src[d] = c;
      }
      return 0;
    }
    if (it == 0) {
      int m[3] = {cur[0], cur[1], cur[2]};
#pragma unroll
      for (int d = 0; d < L::D; ++d) m[d] = min(max(cur[d], a.dlo[d]), a.dhi[d]);
      if (first_face<L>(a, cur, ILBM_BC_USER_2, bd, lo_side)) { src[0] = m[0]; src[1] = m[1]; src[2] = m[2]; return 3; }
      if (first_face<L>(a, cur, ILBM_BC_USER_1, bd, lo_side)) { src[0] = m[0]; src[1] = m[1]; src[2] = m[2]; return 1; }
      if (first_face<L>(a, cur, ILBM_BC_EXT_DIR, bd, lo_side)) { src[0] = m[0]; src[1] = m[1]; src[2] = m[2]; return 2; }
    }
    // foextrap: the last dimension with a foextrap face wins (FilccCell order)
    int dsel = -1;
#pragma unroll
    for (int d = 0; d < L::D; ++d) {
      if (cur[d] < a.dlo[d] && a.bclo[d] == ILBM_BC_FOEXTRAP) dsel = d;
      else if (cur[d] > a.dhi[d] && a.bchi[d] == ILBM_BC_FOEXTRAP) dsel = d;
    }
    if (dsel < 0) break;
    cur[dsel] = (cur[dsel] < a.dlo[dsel]) ? a.dlo[dsel] : a.dhi[dsel];
  }
  src[0] = min(max(g[0], a.dlo[0]), a.dhi[0]);
  src[1] = min(max(g[1], a.dlo[1]), a.dhi[1]);
  src[2] = (L::D == 3) ? min(max(g[2], a.dlo[2]), a.dhi[2]) : 0;
  return 0;
}

// Populations that enter the box from its layer-1 ghost shell are pushed here,
// one thread per ghost cell: the pre-collision boundary value (self-fill: the
// FillPatch rules above on f^n of the domain; caller-filled: the ghost value
// as given), or, for a ghost covered by another box of the level, that cell's
// post-collision value.  Ghosts that are periodic images (self-fill) and
// halfway bounce-back ghosts are left to the owning cells' push.  A ghost cell
// is owned by the slab of its lowest dimension outside the box (periodic
// dimensions excluded in self-fill mode, whose slabs do nothing).
// The work runs in the leading blocks of the k_step launch (it writes only
// slots that no cell's push writes, and reads only f^n), so its strided
// accesses overlap the main stream instead of preceding it.
template <class L, int S>
__device__ __noinline__ void ghost_push(const StepArgs &a, int64_t gid, int64_t gstride) {
  using T = typename Store<S>::T;
  using R = typename Store<S>::R;
  for (int slab = 0; slab < 2 * L::D; ++slab) {
  const int d = slab >> 1, side = slab & 1;
  if (a.self_fill && a.periodic[d]) continue;
  int ext[3], base[3];
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    if (e >= L::D) { ext[e] = 1; base[e] = 0; continue; }
    ext[e] = a.hi[e] - a.lo[e] + 3;
    base[e] = a.lo[e] - 1;
  }
  ext[d] = 1;
  base[d] = side ? a.hi[d] + 1 : a.lo[d] - 1;
  const int64_t n = (int64_t)ext[0] * ext[1] * ext[2];
  T *fo = static_cast<T *>(a.f_out);
  for (int64_t t = gid; t < n; t += gstride) {
    int g[3];
    g[0] = base[0] + (int)(t % ext[0]);
    g[1] = base[1] + (int)((t / ext[0]) % ext[1]);
    g[2] = base[2] + (int)(t / ((int64_t)ext[0] * ext[1]));
    // owner: lowest dimension outside the box whose slab is active (in
    // self-fill mode periodic slabs are skipped)
    int owner = -1;
#pragma unroll
    for (int e = 0; e < L::D; ++e)
      if (owner < 0 && (g[e] < a.lo[e] || g[e] > a.hi[e]) && !(a.self_fill && a.periodic[e]))
        owner = e;
    if (owner != d) continue;
    // classify the ghost against the domain
    bool phys = false, pure_u1 = true;
#pragma unroll
    for (int e = 0; e < L::D; ++e) {
      int sd = 0;
      if (g[e] < a.dlo[e]) sd = -1;
      else if (g[e] > a.dhi[e]) sd = 1;
      if (sd == 0) continue;
      if (a.periodic[e]) {
        pure_u1 = false;
      } else {
        phys = true;
        if ((sd < 0 ? a.bclo[e] : a.bchi[e]) != ILBM_BC_USER_1) pure_u1 = false;
      }
    }
    if (a.self_fill && !phys) continue;  // periodic image: the wrapping push delivers it
    if (phys && pure_u1) continue;       // halfway bounce-back: reflected by the cell
    const int gk = (L::D == 3) ? g[2] : 0;
    // source of the ghost's populations
    int mode;  // 0 copy from src (raw), 1 NEQ boundary formula on src, 2 collide the ghost
    int src[3] = {g[0], g[1], gk}, bd = 0, lo_side = 1, kind = 0;
    if (phys && a.self_fill) {
      kind = ghost_rule<L>(a, g, src, bd, lo_side);
      mode = (kind <= 1) ? 0 : 1;
    } else if (phys) {
      mode = 0;  // caller-filled physical ghost, as given
    } else {
      int gw[3] = {g[0], g[1], gk};
#pragma unroll
      for (int e = 0; e < L::D; ++e)
        if (a.periodic[e]) {
          const int nn = a.dhi[e] - a.dlo[e] + 1;
          gw[e] = a.dlo[e] + (((gw[e] - a.dlo[e]) % nn) + nn) % nn;
        }
      bool covered = false;
      for (int b = 0; b < a.nlb && !covered; ++b)
        covered = gw[0] >= a.lb[b][0] && gw[0] <= a.lb[b][3] && gw[1] >= a.lb[b][1] &&
                  gw[1] <= a.lb[b][4] && (L::D == 2 || (gw[2] >= a.lb[b][2] && gw[2] <= a.lb[b][5]));
      mode = covered ? 2 : 0;  // not covered: coarse-fine ghost, as given
    }
    const int64_t sb = fidx(a, src[0], src[1], L::D == 3 ? src[2] : 0);
    // per-ghost state for the NEQ formula / the collision
    double r64 = 0, u64 = 0, v64 = 0, w64 = 0, rt64 = 0, ut64 = 0, vt64 = 0, wt64 = 0;
    float dr32 = 0, u32 = 0, v32 = 0, w32 = 0, drt32 = 0, ut32 = 0, vt32 = 0, wt32 = 0;
    R gFx = R(0), gFy = R(0), gFz = R(0);
    bool ghf = false;
    if (mode == 1) {
      // applyExtDirMesoscopic / applyFaceMirroredMesoscopic, bc_fill.H:159-261
      const double *bv = lo_side ? a.bvlo[bd] : a.bvhi[bd];
      if (S == ILBM_STORAGE_F64) {
        double rhonp = 0.0, unp = 0.0, vnp = 0.0, wnp = 0.0;
#pragma unroll
        for (int p = 0; p < L::Q; ++p) {
          const double fp = ldf<L, S>(a, sb, p);
          rhonp = X::add(rhonp, fp);
          unp = X::add(unp, X::mul(double(L::cx(p)), fp));
          vnp = X::add(vnp, X::mul(double(L::cy(p)), fp));
          wnp = X::add(wnp, X::mul(double(L::cz(p)), fp));
        }
        rhonp = fmax(rhonp, 1.0e-20);
        r64 = rhonp;
        u64 = X::div(unp, rhonp);
        v64 = X::div(vnp, rhonp);
        w64 = X::div(wnp, rhonp);
        rt64 = bv[0]; ut64 = bv[1]; vt64 = bv[2]; wt64 = bv[3];
        if (kind == 3) {
          rt64 = fmax(1.0e-20, X::sub(X::mul(2.0, bv[0]), r64));
          ut64 = X::sub(X::mul(2.0, bv[1]), u64);
          vt64 = X::sub(X::mul(2.0, bv[2]), v64);
          wt64 = X::sub(X::mul(2.0, bv[3]), w64);
        }
      } else {
        float rr = 0.f, m1 = 0.f, m2 = 0.f, m3 = 0.f;
#pragma unroll
        for (int p = 0; p < L::Q; ++p) {
          const float gp = ldf<L, S>(a, sb, p);
          rr += gp;
          if (L::cx(p)) m1 += float(L::cx(p)) * gp;
          if (L::cy(p)) m2 += float(L::cy(p)) * gp;
          if (L::cz(p)) m3 += float(L::cz(p)) * gp;
        }
        const float rho = fmaxf(1.0f + rr, 1.0e-20f);
        dr32 = rho - 1.0f;
        u32 = m1 / rho; v32 = m2 / rho; w32 = m3 / rho;
        drt32 = float(bv[0]) - 1.0f; ut32 = float(bv[1]); vt32 = float(bv[2]); wt32 = float(bv[3]);
        if (kind == 3) {
          drt32 = fmaxf(1.0e-20f, 2.0f * float(bv[0]) - rho) - 1.0f;
          ut32 = 2.0f * float(bv[1]) - u32;
          vt32 = 2.0f * float(bv[2]) - v32;
          wt32 = 2.0f * float(bv[3]) - w32;
        }
      }
    } else if (mode == 2) {
      load_force<L, R>(a, a.force, g[0], g[1], gk, gFx, gFy, gFz);
      ghf = !(gFx == R(0) && gFy == R(0) && gFz == R(0));
      if (stored_macro_at(a, g[0], g[1], gk)) {
        const int64_t m = midx(a, g[0], g[1], gk);
        if (S == ILBM_STORAGE_F64) {
          r64 = ldm<double>(a.macro_in, m);
          u64 = ldm<double>(a.macro_in, m + a.ms2);
          v64 = ldm<double>(a.macro_in, m + 2 * a.ms2);
          w64 = (L::D == 3) ? ldm<double>(a.macro_in, m + 3 * a.ms2) : 0.0;
        } else {
          dr32 = ldm<float>(a.macro_in, m) - 1.0f;
          u32 = ldm<float>(a.macro_in, m + a.ms2);
          v32 = ldm<float>(a.macro_in, m + 2 * a.ms2);
          w32 = (L::D == 3) ? ldm<float>(a.macro_in, m + 3 * a.ms2) : 0.0f;
        }
      } else if (S == ILBM_STORAGE_F64) {
        double fg[L::Q];
#pragma unroll
        for (int p = 0; p < L::Q; ++p) fg[p] = ldf<L, S>(a, sb, p);
        double px, py, pz;
        load_force<L, double>(a, a.force_prev, g[0], g[1], gk, px, py, pz);
        moments64<L>(fg, px, py, pz, r64, u64, v64, w64);
        if (L::D != 3) w64 = 0.0;
      } else {
        float fg[L::Q];
#pragma unroll
        for (int p = 0; p < L::Q; ++p) fg[p] = ldf<L, S>(a, sb, p);
        float px, py, pz;
        load_force<L, float>(a, a.force_prev, g[0], g[1], gk, px, py, pz);
        moments32<L>(fg, px, py, pz, dr32, u32, v32, w32);
      }
    }
#pragma unroll
    for (int q = 1; q < L::Q; ++q) {
      const int di = g[0] + L::cx(q), dj = g[1] + L::cy(q), dk = gk + L::cz(q);
      if (!in_box(a.lo, a.hi, di, dj, dk)) continue;
      const R fq = ldf<L, S>(a, sb, q);
      R val;
      if (mode == 0) {
        val = fq;
      } else if (mode == 1) {
        if (S == ILBM_STORAGE_F64)
          val = R(X::add(feq64_3<L>(q, rt64, ut64, vt64, wt64),
                         X::sub(double(fq), feq64_3<L>(q, r64, u64, v64, w64))));
        else
          val = R(feqs<L>(q, drt32, ut32, vt32, wt32) + (float(fq) - feqs<L>(q, dr32, u32, v32, w32)));
      } else {
        if (S == ILBM_STORAGE_F64)
          val = R(collide64_one<L>(q, double(fq), feq64<L>(q, r64, u64, v64, w64), a.tau, u64, v64,
                                   w64, double(gFx), double(gFy), double(gFz), ghf));
        else
          val = R(post32<L>(q, float(fq), col32_setup<L>(dr32, u32, v32, w32, a.om32, a.omh32,
                                                         float(gFx), float(gFy), float(gFz))));
      }
      Store<S>::store(fo + fidx(a, di, dj, dk) + q * a.fs2, val, sfac<L, S>(a, q));
    }
  }
  }  // slab
}

// ---------------------------------------------------------------------------
// Main fused kernel
// ---------------------------------------------------------------------------
// occupancy target: 4 resident blocks of 256 threads per SM for the 4-byte and
// 2-byte storage forms of D2Q9/D3Q19 (<= 64 registers), 2 otherwise
template <class L, int S>
struct StepOcc {
  static constexpr int value = (S != ILBM_STORAGE_F64 && L::Q <= 19) ? 4 : 2;
};

// One cell of the level step: load f^n, recover rho^n/u^n, collide, push.
// `edge` selects the checked push plus the completion of ghost-sourced pulls;
// interior cells take the unchecked path.
template <class L, int S>
__device__ __forceinline__ void cell_finish(const StepArgs &a, int i, int j, int k, bool edge,
                                            typename Store<S>::R *f);

template <class L, int S>
__device__ __forceinline__ void cell_update(const StepArgs &a, int i, int j, int k, bool edge) {
  using T = typename Store<S>::T;
  using R = typename Store<S>::R;
  const T *fin = static_cast<const T *>(a.f_in) + fidx(a, i, j, k);
  R f[L::Q];
#pragma unroll
  for (int q = 0; q < L::Q; ++q) f[q] = Store<S>::load(fin + a.loff[q], sfac<L, S>(a, q));
  cell_finish<L, S>(a, i, j, k, edge, f);
}

// The rest of a cell update once its populations f^n are in registers.
template <class L, int S>
__device__ __forceinline__ void cell_finish(const StepArgs &a, int i, int j, int k, bool edge,
                                            typename Store<S>::R *f) {
  using T = typename Store<S>::T;
  using R = typename Store<S>::R;
  const int64_t base = fidx(a, i, j, k);
  R Fx, Fy, Fz;
  load_force<L, R>(a, a.force, i, j, k, Fx, Fy, Fz);

  // per-cell collision state: rho^n, u^n (stored or recovered) and F^n
  double rho64 = 0, u64 = 0, v64 = 0, w64 = 0;
  float drho32 = 0, u32 = 0, v32 = 0, w32 = 0;
  const bool stored = stored_macro_at(a, i, j, k);
  if (S == ILBM_STORAGE_F64) {
    if (stored) {
      const int64_t m = midx(a, i, j, k);
      rho64 = ldm<double>(a.macro_in, m);
      u64 = ldm<double>(a.macro_in, m + a.ms2);
      v64 = ldm<double>(a.macro_in, m + 2 * a.ms2);
      w64 = (L::D == 3) ? ldm<double>(a.macro_in, m + 3 * a.ms2) : 0.0;
    } else {
      double px, py, pz;
      load_force<L, double>(a, a.force_prev, i, j, k, px, py, pz);
      moments64<L>(reinterpret_cast<double *>(f), px, py, pz, rho64, u64, v64, w64);
      if (L::D != 3) w64 = 0.0;
    }
  } else {
    if (stored) {
      const int64_t m = midx(a, i, j, k);
      drho32 = ldm<float>(a.macro_in, m) - 1.0f;
      u32 = ldm<float>(a.macro_in, m + a.ms2);
      v32 = ldm<float>(a.macro_in, m + 2 * a.ms2);
      w32 = (L::D == 3) ? ldm<float>(a.macro_in, m + 3 * a.ms2) : 0.0f;
    } else {
      float px, py, pz;
      load_force<L, float>(a, a.force_prev, i, j, k, px, py, pz);
      moments32<L>(reinterpret_cast<float *>(f), px, py, pz, drho32, u32, v32, w32);
    }
  }
  // the Guo increment is skipped where F == 0 (collide_forced.H:81-83)
  const bool hf = !(Fx == R(0) && Fy == R(0) && Fz == R(0));
  const Col32 c32 = col32_setup<L>(drho32, u32, v32, w32, a.om32, a.omh32, float(Fx), float(Fy),
                                   float(Fz));
  auto post_v = [&](int q, R fq) -> R {
    if (S == ILBM_STORAGE_F64) {
      const double fe = feq64<L>(q, rho64, u64, v64, w64);
      return R(collide64_one<L>(q, double(fq), fe, a.tau, u64, v64, w64, double(Fx),
                                double(Fy), double(Fz), hf));
    } else {
      return R(post32<L>(q, float(fq), c32));
    }
  };

  T *fo = static_cast<T *>(a.f_out);
  T *fob = fo + base;
  // Push: every thread, edge or not, stores f*(y,q) at y + c_q.  For an edge
  // cell some of these land in the ghost layer of f_out, which is scratch
  // (never read); they are fixed up below.
#pragma unroll
  for (int q = 0; q < L::Q; ++q) Store<S>::store(fob + a.doff[q], post_v(q, f[q]), sfac<L, S>(a, q));
  if (!edge) return;
  // Edge fix-up for destinations outside the box: periodic image (self-fill)
  // -> wrapped push; halfway bounce-back wall -> reflected into this cell
  // (f*(x,q) -> f_out(x, q_bar), AdvanceLBMAtLevel.cpp:272-373); anything
  // else leaves the box (the populations entering from that ghost come from
  // k_ghost_push).  The few populations involved are re-collided from a reload.
  const T *fin_c = static_cast<const T *>(a.f_in) + base;
#pragma unroll
  for (int q = 1; q < L::Q; ++q) {
    int di = i + L::cx(q), dj = j + L::cy(q), dk = k + L::cz(q);
    if (in_box(a.lo, a.hi, di, dj, dk)) continue;
    const int dd[3] = {di, dj, dk};
    bool phys = false, pure_u1 = true;
#pragma unroll
    for (int e = 0; e < L::D; ++e) {
      int sd = 0;
      if (dd[e] < a.dlo[e]) sd = -1;
      else if (dd[e] > a.dhi[e]) sd = 1;
      if (sd == 0) continue;
      if (a.periodic[e]) {
        pure_u1 = false;
      } else {
        phys = true;
        if ((sd < 0 ? a.bclo[e] : a.bchi[e]) != ILBM_BC_USER_1) pure_u1 = false;
      }
    }
    T *dst;
    if (phys) {
      if (!pure_u1) continue;
      dst = fob + a.loff[opposite<L>(q)];
    } else if (a.self_fill) {
      if (L::cx(q) != 0 && (di < a.dlo[0] || di > a.dhi[0])) di = (di < a.dlo[0]) ? a.dhi[0] : a.dlo[0];
      if (L::cy(q) != 0 && (dj < a.dlo[1] || dj > a.dhi[1])) dj = (dj < a.dlo[1]) ? a.dhi[1] : a.dlo[1];
      if (L::D == 3 && L::cz(q) != 0 && (dk < a.dlo[2] || dk > a.dhi[2]))
        dk = (dk < a.dlo[2]) ? a.dhi[2] : a.dlo[2];
      dst = fo + fidx(a, di, dj, dk) + (int64_t)q * a.fs2;
    } else {
      continue;  // another box: its ghost shell push delivers
    }
    const R fq = Store<S>::load(fin_c + a.loff[q], sfac<L, S>(a, q));
    // (w_q = w_{q_bar}: the FP16 storage factor is the same for a reflection)
    Store<S>::store(dst, post_v(q, fq), sfac<L, S>(a, q));
  }
}

// Main kernel: one thread per cell of a row segment (rows on a box face run
// the checked push as a whole; only the two x-edge cells of a row diverge).
// the edge fix-up is needed only on faces whose outgoing populations come
// back into the box (self-filled periodic: wrapped; user_1: reflected)
template <class L>
__device__ __forceinline__ bool needs_fixup(const StepArgs &a, int i, int j, int k) {
  return (i == a.lo[0] && a.act_lo[0]) || (i == a.hi[0] && a.act_hi[0]) ||
         (j == a.lo[1] && a.act_lo[1]) || (j == a.hi[1] && a.act_hi[1]) ||
         (L::D == 3 && ((k == a.lo[2] && a.act_lo[2]) || (k == a.hi[2] && a.act_hi[2])));
}

// Row segments that need none of the per-cell tests of cell_update take a
// lean path: no face of the segment returns outgoing populations (wrap /
// reflect), no cell reads stored macro fields, none lies in the skip box,
// and the force is of one kind over the whole segment.  The kind is the same
// for every thread of a block (one block = one row segment), so the branch
// does not diverge.
enum SegKind { SEG_GENERAL = 0, SEG_SKIP = 1, SEG_ZERO = 2, SEG_UNIFORM = 3, SEG_ARRAYS = 4 };

template <class L>
__device__ __forceinline__ int seg_kind(const StepArgs &a, int i0, int i1, int j, int k) {
  if (a.use_skip && j >= a.slo[1] && j <= a.shi[1] &&
      (L::D == 2 || (k >= a.slo[2] && k <= a.shi[2]))) {
    if (i0 >= a.slo[0] && i1 <= a.shi[0]) return SEG_SKIP;
    if (!(i1 < a.slo[0] || i0 > a.shi[0])) return SEG_GENERAL;
  }
  if ((j == a.lo[1] && a.act_lo[1]) || (j == a.hi[1] && a.act_hi[1])) return SEG_GENERAL;
  if (L::D == 3 && ((k == a.lo[2] && a.act_lo[2]) || (k == a.hi[2] && a.act_hi[2])))
    return SEG_GENERAL;
  if ((i0 == a.lo[0] && a.act_lo[0]) || (i1 == a.hi[0] && a.act_hi[0])) return SEG_GENERAL;
  if (a.macro_in) {
    if (!a.use_mbox) return SEG_GENERAL;
    if (j >= a.mblo[1] && j <= a.mbhi[1] && k >= a.mblo[2] && k <= a.mbhi[2] &&
        !(i1 < a.mblo[0] || i0 > a.mbhi[0]))
      return SEG_GENERAL;
  }
  if (a.force == nullptr || a.force_prev == nullptr) {
    if (a.force != nullptr || a.force_prev != nullptr) return SEG_GENERAL;
    return a.use_uniform ? SEG_UNIFORM : SEG_ZERO;
  }
  // force arrays: zero outside [flo, fhi] (F^n and F^{n-1} alike)
  if (j < a.flo[1] || j > a.fhi[1] || (L::D == 3 && (k < a.flo[2] || k > a.fhi[2])) ||
      i1 < a.flo[0] || i0 > a.fhi[0])
    return SEG_ZERO;
  if (i0 >= a.flo[0] && i1 <= a.fhi[0]) return SEG_ARRAYS;
  return SEG_GENERAL;
}

// One cell of a lean row segment: the same arithmetic as cell_update with
// edge = false on rho^n, u^n recovered from f^n and F^{n-1}.
template <class L, int S, int K>
__device__ __forceinline__ void cell_fast(const StepArgs &a, int i, int j, int k) {
  using T = typename Store<S>::T;
  using R = typename Store<S>::R;
  const int64_t base = fidx(a, i, j, k);
  const T *fin = static_cast<const T *>(a.f_in) + base;
  R f[L::Q];
#pragma unroll
  for (int q = 0; q < L::Q; ++q) f[q] = Store<S>::load(fin + a.loff[q], sfac<L, S>(a, q));
  R Fx = R(0), Fy = R(0), Fz = R(0), px = R(0), py = R(0), pz = R(0);
  if (K == SEG_ARRAYS) {
    const int64_t m = midx(a, i, j, k);
    const R *F = static_cast<const R *>(a.force);
    const R *P = static_cast<const R *>(a.force_prev);
    Fx = F[m];
    Fy = F[m + a.ms2];
    px = P[m];
    py = P[m + a.ms2];
    if (L::D == 3) {
      Fz = F[m + 2 * a.ms2];
      pz = P[m + 2 * a.ms2];
    }
  } else if (K == SEG_UNIFORM) {
    Fx = px = R(a.uf[0]);
    Fy = py = R(a.uf[1]);
    Fz = pz = R(a.uf[2]);
  }
  T *fob = static_cast<T *>(a.f_out) + base;
  if (S == ILBM_STORAGE_F64) {
    double rho, u, v, w;
    moments64<L>(reinterpret_cast<double *>(f), double(px), double(py), double(pz), rho, u, v, w);
    if (L::D != 3) w = 0.0;
    const bool hf = !(Fx == R(0) && Fy == R(0) && Fz == R(0));
#pragma unroll
    for (int q = 0; q < L::Q; ++q)
      Store<S>::store(fob + a.doff[q],
                      R(collide64_one<L>(q, double(f[q]), feq64<L>(q, rho, u, v, w), a.tau, u, v, w,
                                         double(Fx), double(Fy), double(Fz), hf)),
                      sfac<L, S>(a, q));
  } else {
    float drho, u, v, w;
    moments32<L>(reinterpret_cast<float *>(f), float(px), float(py), float(pz), drho, u, v, w);
    const Col32 c = col32_setup<L>(drho, u, v, w, a.om32, a.omh32, float(Fx), float(Fy), float(Fz));
#pragma unroll
    for (int q = 0; q < L::Q; ++q)
      Store<S>::store(fob + a.doff[q], R(post32<L>(q, float(f[q]), c)), sfac<L, S>(a, q));
  }
}

// The first `ghost_slices` z-slices of the grid push the ghost shell's
// populations (ghost_push); the rest run one cell per thread.
template <class L, int S>
__global__ void __launch_bounds__(256, StepOcc<L, S>::value) k_step(const __grid_constant__ StepArgs a) {
  if ((int)blockIdx.z < a.ghost_slices) {
    const int64_t blk = blockIdx.x + (int64_t)gridDim.x * (blockIdx.y + (int64_t)gridDim.y * blockIdx.z);
    ghost_push<L, S>(a, blk * blockDim.x + threadIdx.x,
                     (int64_t)a.ghost_slices * gridDim.x * gridDim.y * blockDim.x);
    return;
  }
  const int i0 = a.rlo[0] + blockIdx.x * blockDim.x;
  const int i = i0 + threadIdx.x;
  const int j = a.rlo[1] + blockIdx.y;
  const int k = a.rlo[2] + (int)blockIdx.z - a.ghost_slices;
  const int kind = seg_kind<L>(a, i0, min(i0 + (int)blockDim.x - 1, a.rhi[0]), j, k);
  if (i > a.rhi[0] || kind == SEG_SKIP) return;
  if (kind == SEG_ZERO) {
    cell_fast<L, S, SEG_ZERO>(a, i, j, k);
  } else if (kind == SEG_UNIFORM) {
    cell_fast<L, S, SEG_UNIFORM>(a, i, j, k);
  } else if (kind == SEG_ARRAYS) {
    cell_fast<L, S, SEG_ARRAYS>(a, i, j, k);
  } else {
    if (a.use_skip && in_box(a.slo, a.shi, i, j, k)) return;
    cell_update<L, S>(a, i, j, k, needs_fixup<L>(a, i, j, k));
  }
}

// ---------------------------------------------------------------------------
// Batched level step: many independent cases (each one box = its level
// domain, self-filled ghosts) in one persistent launch.  Blocks walk a tile
// table of row segments and ghost-push chunks over all cases; the arguments
// of a tile's case are copied to shared memory, so the per-direction offsets
// stay on chip and cannot alias the population stores.
// ---------------------------------------------------------------------------
// the batched step's occupancy target: 5 blocks of 256 (48 registers) for
// D2Q9 in the 4- and 2-byte forms (measured 5% faster on the 64-case D2Q9
// batch than 4), as k_step otherwise
template <class L, int S>
struct BatchOcc {
  static constexpr int value = (S != ILBM_STORAGE_F64 && L::Q <= 9) ? 5 : StepOcc<L, S>::value;
};

template <class L, int S>
__global__ void __launch_bounds__(256, BatchOcc<L, S>::value)
    k_step_batch(const StepArgs *__restrict__ args, const StepTile *__restrict__ tiles, int ntiles,
                 const int *steps, const int *limit) {
  __shared__ StepArgs sa;
  int cur = -1;  // every thread walks the same tiles, so this stays block-uniform
  // strided over the table (block b takes entries b, b + gridDim.x, ...),
  // which the batch lays out so that the blocks in flight stream through
  // neighbouring rows together (a contiguous run of rows per block measured
  // 2.2x slower: the push stores' split lines no longer meet in L2) while a
  // block keeps to one case; c = -1 marks a filler entry
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const StepTile tl = tiles[t];
    if (tl.c < 0 || steps[tl.c] >= limit[tl.c]) continue;  // filler, or a case that has taken all its steps
    if (tl.c != cur) {
      __syncthreads();  // every thread is done with the previous case's arguments
      const int *src = reinterpret_cast<const int *>(args + tl.c);
      int *dst = reinterpret_cast<int *>(&sa);
      for (int w = threadIdx.x; w < (int)(sizeof(StepArgs) / sizeof(int)); w += blockDim.x)
        dst[w] = src[w];
      __syncthreads();
      cur = tl.c;
    }
    if (tl.i0 < 0) {
      ghost_push<L, S>(sa, (int64_t)(-1 - tl.i0) * blockDim.x + threadIdx.x,
                       (int64_t)tl.j * blockDim.x);
      continue;
    }
    // lean row segments as in k_step (a skip box, which single-level cases
    // do not have, stays on the general path as before)
    const int i = tl.i0 + threadIdx.x;
    const int kind = seg_kind<L>(sa, tl.i0, min(tl.i0 + (int)blockDim.x - 1, sa.hi[0]), tl.j, tl.k);
    if (i > sa.hi[0]) continue;
    if (kind == SEG_ZERO)
      cell_fast<L, S, SEG_ZERO>(sa, i, tl.j, tl.k);
    else if (kind == SEG_UNIFORM)
      cell_fast<L, S, SEG_UNIFORM>(sa, i, tl.j, tl.k);
    else if (kind == SEG_ARRAYS)
      cell_fast<L, S, SEG_ARRAYS>(sa, i, tl.j, tl.k);
    else
      cell_update<L, S>(sa, i, tl.j, tl.k, needs_fixup<L>(sa, i, tl.j, tl.k));
  }
}



// ---------------------------------------------------------------------------
// Macro pass (calculateMacroForcing) and equilibrium initialisation
// ---------------------------------------------------------------------------
template <class L, int S>
__global__ void __launch_bounds__(256) k_macro(StepArgs a, int rlo0, int rlo1, int rlo2,
                                               int rhi0, void *macro_out) {
  using R = typename Store<S>::R;
  const int i = rlo0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = rlo1 + blockIdx.y;
  const int k = rlo2 + blockIdx.z;
  if (i > rhi0) return;
  const int64_t base = fidx(a, i, j, k);
  R f[L::Q];
#pragma unroll
  for (int q = 0; q < L::Q; ++q) f[q] = ldf<L, S>(a, base, q);
  R Fx, Fy, Fz;
  load_force<L, R>(a, a.force, i, j, k, Fx, Fy, Fz);
  R *mo = static_cast<R *>(macro_out);
  const int64_t m = midx(a, i, j, k);
  if (S == ILBM_STORAGE_F64) {
    double rho, u, v, w;
    moments64<L>(reinterpret_cast<double *>(f), Fx, Fy, Fz, rho, u, v, w);
    mo[m] = rho;
    mo[m + a.ms2] = u;
    mo[m + 2 * a.ms2] = v;
    mo[m + 3 * a.ms2] = w;
  } else {
    float drho, u, v, w;
    moments32<L>(reinterpret_cast<float *>(f), Fx, Fy, Fz, drho, u, v, w);
    mo[m] = 1.0f + drho;
    mo[m + a.ms2] = u;
    mo[m + 2 * a.ms2] = v;
    mo[m + 3 * a.ms2] = w;
  }
}

// InitEquilibrium, AmrCoreLBM.cpp:2117-2164, over the allocated f box
template <class L, int S>
__global__ void __launch_bounds__(256) k_init_eq(StepArgs a, int ng) {
  using T = typename Store<S>::T;
  const int i = a.lo[0] - ng + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = a.lo[1] - ng + blockIdx.y;
  const int k = (L::D == 3) ? a.lo[2] - ng + blockIdx.z : 0;
  if (i > a.hi[0] + ng) return;
  const int64_t m = midx(a, i, j, k);
  const int64_t b = fidx(a, i, j, k);
  T *f1 = static_cast<T *>(const_cast<void *>(a.f_in));
  T *f2 = static_cast<T *>(a.f_out);
  if (S == ILBM_STORAGE_F64) {
    const double r = fmax(ldm<double>(a.macro_in, m), 1.e-12);
    const double u0 = ldm<double>(a.macro_in, m + a.ms2);
    const double v0 = ldm<double>(a.macro_in, m + 2 * a.ms2);
    const double w0 = (L::D == 3) ? ldm<double>(a.macro_in, m + 3 * a.ms2) : 0.0;
#pragma unroll
    for (int q = 0; q < L::Q; ++q) {
      const double fe = feq64_3<L>(q, r, u0, v0, w0);
      reinterpret_cast<double *>(f1)[b + q * a.fs2] = fe;
      reinterpret_cast<double *>(f2)[b + q * a.fs2] = fe;
    }
  } else {
    const float r = fmaxf(ldm<float>(a.macro_in, m), 1.e-12f);
    const float u0 = ldm<float>(a.macro_in, m + a.ms2);
    const float v0 = ldm<float>(a.macro_in, m + 2 * a.ms2);
    const float w0 = (L::D == 3) ? ldm<float>(a.macro_in, m + 3 * a.ms2) : 0.0f;
#pragma unroll
    for (int q = 0; q < L::Q; ++q) {
      const float ge = feqs<L>(q, r - 1.0f, u0, v0, w0);
      Store<S>::store(f1 + b + q * a.fs2, ge, sfac<L, S>(a, q));
      Store<S>::store(f2 + b + q * a.fs2, ge, sfac<L, S>(a, q));
    }
  }
}

// ---------------------------------------------------------------------------
// Band macro for the immersed boundary: rho, u, v, w (FP64) on the cells of
// the IB support band, including up to two ghost layers outside the domain.
// Valid cells: from macro_in, or from f^n and F^{n-1} (the value the
// reference's macro pass stored).  Ghost cells: FillPatchMacro semantics
// (periodic image, foextrap, macroBcFill: user_2 mirrored state, user_1 /
// ext_dir prescribed state; Source/BC/bc_fill.H:69-142, 263-301).
// ---------------------------------------------------------------------------
template <class L, int S>
__device__ void macro_at(const StepArgs &a, int i, int j, int k, double *m4) {
  if (stored_macro_at(a, i, j, k)) {
    const int64_t m = midx(a, i, j, k);
    if (S == ILBM_STORAGE_F64) {
      m4[0] = ldm<double>(a.macro_in, m);
      m4[1] = ldm<double>(a.macro_in, m + a.ms2);
      m4[2] = ldm<double>(a.macro_in, m + 2 * a.ms2);
      m4[3] = (L::D == 3) ? ldm<double>(a.macro_in, m + 3 * a.ms2) : 0.0;
    } else {
      m4[0] = ldm<float>(a.macro_in, m);
      m4[1] = ldm<float>(a.macro_in, m + a.ms2);
      m4[2] = ldm<float>(a.macro_in, m + 2 * a.ms2);
      m4[3] = (L::D == 3) ? ldm<float>(a.macro_in, m + 3 * a.ms2) : 0.0;
    }
    return;
  }
  const int64_t b = fidx(a, i, j, k);
  if (S == ILBM_STORAGE_F64) {
    double f[L::Q];
#pragma unroll
    for (int q = 0; q < L::Q; ++q) f[q] = ldf<L, S>(a, b, q);
    double px, py, pz;
    load_force<L, double>(a, a.force_prev, i, j, k, px, py, pz);
    moments64<L>(f, px, py, pz, m4[0], m4[1], m4[2], m4[3]);
    if (L::D != 3) m4[3] = 0.0;
  } else {
    float g[L::Q];
#pragma unroll
    for (int q = 0; q < L::Q; ++q) g[q] = ldf<L, S>(a, b, q);
    float px, py, pz, drho, u, v, w;
    load_force<L, float>(a, a.force_prev, i, j, k, px, py, pz);
    moments32<L>(g, px, py, pz, drho, u, v, w);
    m4[0] = 1.0 + double(drho);
    m4[1] = u;
    m4[2] = v;
    m4[3] = (L::D == 3) ? double(w) : 0.0;
  }
}

template <class L, int S>
__device__ __forceinline__ void band_macro_cell(const StepArgs &a, int blo0, int blo1, int blo2,
                                                int bn0, int bn1, int64_t nb, int64_t t,
                                                double *EV, double *RHO) {
  {
    int g[3];
    g[0] = blo0 + (int)(t % bn0);
    g[1] = blo1 + (int)((t / bn0) % bn1);
    g[2] = blo2 + (int)(t / ((int64_t)bn0 * bn1));
    double m4[4];
    bool in = in_domain<L>(a, g[0], g[1], g[2]);
    if (in || (a.macro_in && !a.self_fill)) {
      // caller-filled macros carry their own ghost values
      macro_at<L, S>(a, g[0], g[1], L::D == 3 ? g[2] : 0, m4);
    } else {
      int src[3], bd = 0, lo_side = 1;
      const int kind = ghost_rule<L>(a, g, src, bd, lo_side);
      macro_at<L, S>(a, src[0], src[1], L::D == 3 ? src[2] : 0, m4);
      const double *bv = lo_side ? a.bvlo[bd] : a.bvhi[bd];
      if (kind == 3) {
        m4[0] = fmax(1.0e-20, X::sub(X::mul(2.0, bv[0]), m4[0]));
        m4[1] = X::sub(X::mul(2.0, bv[1]), m4[1]);
        m4[2] = X::sub(X::mul(2.0, bv[2]), m4[2]);
        m4[3] = X::sub(X::mul(2.0, bv[3]), m4[3]);
      } else if (kind == 1 || kind == 2) {
        m4[0] = bv[0];
        m4[1] = bv[1];
        m4[2] = bv[2];
        m4[3] = bv[3];
      }
    }
    EV[t] = m4[1];
    EV[t + nb] = m4[2];
    EV[t + 2 * nb] = (L::D == 3) ? m4[3] : 0.0;
    RHO[t] = m4[0];
  }
}

template <class L, int S>
__global__ void __launch_bounds__(256) k_band_macro(StepArgs a, int blo0, int blo1, int blo2,
                                                    int bn0, int bn1, int bn2, double *EV,
                                                    double *RHO) {
  const int64_t nb = (int64_t)bn0 * bn1 * bn2;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nb;
       t += (int64_t)gridDim.x * blockDim.x)
    band_macro_cell<L, S>(a, blo0, blo1, blo2, bn0, bn1, nb, t, EV, RHO);
}

// the band cells of a list (band indices): the cells a fixed body's stencils
// reach, which are all that its interpolation and export read
template <class L, int S>
__global__ void __launch_bounds__(256) k_band_macro_list(StepArgs a, int blo0, int blo1, int blo2,
                                                         int bn0, int bn1, int bn2,
                                                         const int64_t *__restrict__ cells,
                                                         int ncells, double *EV, double *RHO) {
  const int64_t nb = (int64_t)bn0 * bn1 * bn2;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < ncells; r += gridDim.x * blockDim.x)
    band_macro_cell<L, S>(a, blo0, blo1, blo2, bn0, bn1, nb, cells[r], EV, RHO);
}

// one block of kItemTile threads per band tile (case, first cell)
template <class L, int S>
__global__ void __launch_bounds__(kItemTile) k_band_macro_batch(const StepArgs *args,
                                                                const BandDesc *bands,
                                                                const ItemRef *tiles, int ntiles,
                                                                const int *steps, const int *limit) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const ItemRef e = tiles[t];
    const int c = e.c;
    if (steps[c] >= limit[c]) continue;
    const BandDesc &b = bands[c];
    const int64_t u = (int64_t)e.u + threadIdx.x;
    if (u >= b.nb) continue;
    band_macro_cell<L, S>(args[c], b.blo[0], b.blo[1], b.blo[2], b.bn[0], b.bn[1], b.nb, u, b.EV,
                          b.RHO);
    if (b.EFI) b.EFI[u] = b.EFI[u + b.nb] = b.EFI[u + 2 * b.nb] = 0.0;  // spread target of this step
  }
}

// Band macro of a level held in several boxes (caller-filled ghosts), the
// EulerVel of IBMarkerDF::update_forcing (Source/IBM/IBMarkerDF.cpp:1541-1566)
// followed by its FillBoundary (:702-703): a band cell takes rho, u from the
// box whose valid region holds it; a cell that no box holds (a coarse-fine or
// physical ghost of the level) takes the caller-filled ghost value of the
// first box whose grown arrays reach it; a cell that none reaches gets the
// reference's initial EulerVel, zero velocity (and unit density).
template <class L>
__device__ __forceinline__ bool valid_at(const StepArgs &a, int i, int j, int k) {
  return i >= a.lo[0] && i <= a.hi[0] && j >= a.lo[1] && j <= a.hi[1] &&
         (L::D == 2 || (k >= a.lo[2] && k <= a.hi[2]));
}

// the cell can be read from the box's grown arrays: macro_in grown by
// ngrow_m, else f_in and force_prev grown by the smaller of their widths
template <class L>
__device__ __forceinline__ bool readable_at(const StepArgs &a, int i, int j, int k) {
  const int g[3] = {i, j, k};
#pragma unroll
  for (int d = 0; d < L::D; ++d) {
    const int gm = a.lo[d] - a.mgl[d], gf = a.lo[d] - a.fgl[d];
    const int w = a.macro_in ? gm : min(gm, gf);
    if (g[d] < a.lo[d] - w || g[d] > a.hi[d] + w) return false;
  }
  return true;
}

template <class L, int S>
__global__ void __launch_bounds__(256) k_band_macro_boxes(const StepArgs *__restrict__ args, int nargs,
                                                          int blo0, int blo1, int blo2, int bn0,
                                                          int bn1, int bn2, double *EV, double *RHO) {
  const int64_t nb = (int64_t)bn0 * bn1 * bn2;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nb;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int i = blo0 + (int)(t % bn0);
    const int j = blo1 + (int)((t / bn0) % bn1);
    const int k = (L::D == 3) ? blo2 + (int)(t / ((int64_t)bn0 * bn1)) : 0;
    int src = -1;
    for (int b = 0; b < nargs && src < 0; ++b)
      if (valid_at<L>(args[b], i, j, k)) src = b;
    for (int b = 0; b < nargs && src < 0; ++b)
      if (readable_at<L>(args[b], i, j, k)) src = b;
    double m4[4] = {1.0, 0.0, 0.0, 0.0};
    if (src >= 0) macro_at<L, S>(args[src], i, j, k, m4);
    EV[t] = m4[1];
    EV[t + nb] = m4[2];
    EV[t + 2 * nb] = (L::D == 3) ? m4[3] : 0.0;
    RHO[t] = m4[0];
  }
}

template <class L, int S>
static int launch_band_macro_boxes(ilbm_ctx *ctx, const StepArgs *d_args, int nargs,
                                   const int *blo, const int *bn, double *EV, double *RHO,
                                   cudaStream_t st) {
  const int64_t nb = (int64_t)bn[0] * bn[1] * bn[2];
  const int blocks = (int)std::min<int64_t>((nb + 255) / 256, 2048);
  k_band_macro_boxes<L, S><<<blocks, 256, 0, st>>>(d_args, nargs, blo[0], blo[1], blo[2], bn[0],
                                                   bn[1], bn[2], EV, RHO);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "band macro launch");
  return ILBM_OK;
}

template <class L, int S>
static int launch_band_macro(ilbm_ctx *ctx, const StepArgs &a, const int *blo, const int *bn,
                             double *EV, double *RHO, cudaStream_t st) {
  const int64_t nb = (int64_t)bn[0] * bn[1] * bn[2];
  const int blocks = (int)std::min<int64_t>((nb + 255) / 256, 2048);
  k_band_macro<L, S><<<blocks, 256, 0, st>>>(a, blo[0], blo[1], blo[2], bn[0], bn[1], bn[2], EV,
                                              RHO);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "band macro launch");
  return ILBM_OK;
}

template <class L, int S>
static int launch_band_macro_list(ilbm_ctx *ctx, const StepArgs &a, const int *blo, const int *bn,
                                  const int64_t *cells, int ncells, double *EV, double *RHO,
                                  cudaStream_t st) {
  if (ncells <= 0) return ILBM_OK;
  const int blocks = std::min((ncells + 255) / 256, 2048);
  k_band_macro_list<L, S><<<blocks, 256, 0, st>>>(a, blo[0], blo[1], blo[2], bn[0], bn[1], bn[2],
                                                   cells, ncells, EV, RHO);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "band macro launch");
  return ILBM_OK;
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static int fill_args(const ilbm_ctx *ctx, const ilbm_box &b, const ilbm_level_params *p,
                     StepArgs &a) {
  std::memset(&a, 0, sizeof(a));
  const int D = ctx->dim;
  for (int d = 0; d < 3; ++d) {
    a.lo[d] = (d < D) ? b.lo[d] : 0;
    a.hi[d] = (d < D) ? b.hi[d] : 0;
    a.fgl[d] = (d < D) ? b.lo[d] - b.ngrow_f : 0;
    a.mgl[d] = (d < D) ? b.lo[d] - b.ngrow_m : 0;
  }
  for (int d = 0; d < 3; ++d) {
    a.rlo[d] = a.lo[d];
    a.rhi[d] = a.hi[d];
  }
  a.use_skip = 0;
  a.fs0 = b.fstride[0];
  a.fs1 = b.fstride[1];
  a.fs2 = b.fstride[2];
  a.ms0 = b.mstride[0];
  a.ms1 = b.mstride[1];
  a.ms2 = b.mstride[2];
  a.f_in = b.f_in;
  a.f_out = b.f_out;
  {
    static const int cx9[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
    static const int cy9[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
    static const int cx19[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
    static const int cy19[19] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
    static const int cz19[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
    for (int q = 0; q < ctx->q; ++q) {
      int cx = 0, cy = 0, cz = 0;
      if (ctx->q == 9) { cx = cx9[q]; cy = cy9[q]; }
      else if (ctx->q == 19) { cx = cx19[q]; cy = cy19[q]; cz = cz19[q]; }
      else { cx = Lat<27>::cx(q); cy = Lat<27>::cy(q); cz = Lat<27>::cz(q); }
      const int64_t lo = (int64_t)q * b.fstride[2];
      const int64_t dof = lo + cx + (int64_t)cy * b.fstride[0] + (int64_t)cz * b.fstride[1];
      if (lo > INT32_MAX || dof > INT32_MAX || dof < INT32_MIN) {
        set_error("box too large for 32-bit per-direction offsets (Q * component stride >= 2^31)");
        return ILBM_ERR_RANGE;
      }
      a.loff[q] = (int32_t)lo;
      a.doff[q] = (int32_t)dof;
    }
  }
  a.macro_in = b.macro_in;
  a.force = b.force;
  a.force_prev = b.force_prev;
  if (p) {
    for (int d = 0; d < 3; ++d) {
      a.dlo[d] = (d < D) ? p->domain_lo[d] : 0;
      a.dhi[d] = (d < D) ? p->domain_hi[d] : 0;
      a.periodic[d] = (d < D) ? p->periodic[d] : 0;
      a.bclo[d] = p->bc_lo[d];
      a.bchi[d] = p->bc_hi[d];
      for (int c = 0; c < 4; ++c) {
        a.bvlo[d][c] = p->bc_val_lo[d][c];
        a.bvhi[d][c] = p->bc_val_hi[d][c];
      }
      // never read force outside its allocation
      a.flo[d] = (d < D) ? std::max(p->force_lo[d], b.lo[d] - b.ngrow_m) : 0;
      a.fhi[d] = (d < D) ? std::min(p->force_hi[d], b.hi[d] + b.ngrow_m) : 0;
    }
    a.tau = p->tau;
    a.om32 = float(1.0 / p->tau);
    a.omh32 = float(1.0 - 0.5 / p->tau);
    a.self_fill = (p->ghost_mode == ILBM_GHOST_SELF);
    a.use_uniform = p->use_uniform_force;
    for (int d = 0; d < 3; ++d) a.uf[d] = p->uniform_force[d];
    a.f16_scale = (p->f16_scale > 0) ? float(p->f16_scale) : 1024.0f;
    // faces that send outgoing populations back into the box: domain faces
    // that are periodic with self-filled ghosts (wrapped push) or user_1
    // (halfway bounce-back); every other face leaves them to ghost_push
    for (int d = 0; d < D; ++d) {
      const bool plo = a.periodic[d] ? a.self_fill : (a.bclo[d] == ILBM_BC_USER_1);
      const bool phi = a.periodic[d] ? a.self_fill : (a.bchi[d] == ILBM_BC_USER_1);
      a.act_lo[d] = (a.lo[d] == a.dlo[d]) && plo;
      a.act_hi[d] = (a.hi[d] == a.dhi[d]) && phi;
    }
    if (p->ghost_mode == ILBM_GHOST_CALLER) {
      if (p->nlevel_boxes > kMaxLevelBoxes) {
        set_error("level has more boxes than one call supports (64); split the call");
        return ILBM_ERR_RANGE;
      }
      a.nlb = p->nlevel_boxes;
      for (int n = 0; n < a.nlb; ++n)
        for (int c = 0; c < 6; ++c) a.lb[n][c] = p->level_boxes[6 * n + c];
    }
  } else {
    a.f16_scale = 1024.0f;
  }
  return ILBM_OK;
}

// ghost cells whose populations ghost_push delivers (0 when every face is a
// self-filled periodic one)
template <class L>
static int64_t ghost_work(const StepArgs &a) {
  int64_t n = 0;
  for (int d = 0; d < L::D; ++d) {
    if (a.self_fill && a.periodic[d]) continue;
    int64_t s = 1;
    for (int e = 0; e < L::D; ++e)
      if (e != d) s *= (a.hi[e] - a.lo[e] + 3);
    n += 2 * s;
  }
  return n;
}

// k_step over [rlo, rhi] (minus the skip box), with the ghost shell push in
// leading z-slices when with_ghosts is set
template <class L, int S>
static void launch_cells(ilbm_ctx *ctx, const StepArgs &a_in, cudaStream_t st, bool with_ghosts) {
  StepArgs a = a_in;
  const int nx = a.rhi[0] - a.rlo[0] + 1, ny = a.rhi[1] - a.rlo[1] + 1;
  const int nz = (L::D == 3) ? a.rhi[2] - a.rlo[2] + 1 : 1;
  if (nx <= 0 || ny <= 0 || nz <= 0) return;
  const int bx = nx >= 256 ? 256 : ((nx + 31) / 32) * 32;
  const int gx = (nx + bx - 1) / bx;
  a.ghost_slices = 0;
  if (with_ghosts) {
    // about one ghost cell per thread
    const int64_t per_slice = (int64_t)gx * ny * bx;
    const int64_t w = ghost_work<L>(a);
    if (w > 0) a.ghost_slices = (int)std::min<int64_t>(64, (w + per_slice - 1) / per_slice);
  }
  dim3 grid(gx, ny, nz + a.ghost_slices);
  k_step<L, S><<<grid, bx, 0, st>>>(a);
  ctx->launches++;
}

template <class L, int S>
static int launch_step(ilbm_ctx *ctx, const StepArgs &a, const ilbm_level_params *p) {
  (void)p;
  launch_cells<L, S>(ctx, a, ctx->stream, true);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "level step launch");
  return ILBM_OK;
}

// the cells [a.rlo, a.rhi] of a level step, with the ghost-shell push or not
template <class L, int S>
static int launch_step_part(ilbm_ctx *ctx, const StepArgs &a, bool with_ghosts) {
  launch_cells<L, S>(ctx, a, ctx->stream, with_ghosts);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "level step launch");
  return ILBM_OK;
}

// Level step whose band [blo,bhi] waits for `band_ready` (recorded on another
// stream): ghost push and every cell outside the band run first, then the band.
template <class L, int S>
static int launch_step_split(ilbm_ctx *ctx, const StepArgs &a, const int *blo, const int *bhi,
                             cudaEvent_t band_ready) {
  StepArgs outer = a;
  outer.use_skip = 1;
  for (int d = 0; d < 3; ++d) {
    outer.slo[d] = blo[d];
    outer.shi[d] = bhi[d];
  }
  launch_cells<L, S>(ctx, outer, ctx->stream, true);
  cudaError_t e = cudaStreamWaitEvent(ctx->stream, band_ready, 0);
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamWaitEvent");
  StepArgs inner = a;
  for (int d = 0; d < 3; ++d) {
    inner.rlo[d] = blo[d];
    inner.rhi[d] = bhi[d];
  }
  launch_cells<L, S>(ctx, inner, ctx->stream, false);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "level step launch");
  return ILBM_OK;
}

template <class L, int S>
static int launch_macro(ilbm_ctx *ctx, const StepArgs &a, const int *rlo, const int *rhi,
                        void *macro_out) {
  const int nx = rhi[0] - rlo[0] + 1, ny = rhi[1] - rlo[1] + 1;
  const int nz = (L::D == 3) ? rhi[2] - rlo[2] + 1 : 1;
  if (nx <= 0 || ny <= 0 || nz <= 0) return ILBM_OK;
  const int bx = nx >= 256 ? 256 : ((nx + 31) / 32) * 32;
  dim3 grid((nx + bx - 1) / bx, ny, nz);
  k_macro<L, S><<<grid, bx, 0, ctx->stream>>>(a, rlo[0], rlo[1], (L::D == 3) ? rlo[2] : 0,
                                              rhi[0], macro_out);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "macro launch");
  return ILBM_OK;
}

template <class L, int S>
static int launch_init(ilbm_ctx *ctx, const StepArgs &a, int ng) {
  const int nx = a.hi[0] - a.lo[0] + 1 + 2 * ng, ny = a.hi[1] - a.lo[1] + 1 + 2 * ng;
  const int nz = (L::D == 3) ? a.hi[2] - a.lo[2] + 1 + 2 * ng : 1;
  const int bx = nx >= 256 ? 256 : ((nx + 31) / 32) * 32;
  dim3 grid((nx + bx - 1) / bx, ny, nz);
  k_init_eq<L, S><<<grid, bx, 0, ctx->stream>>>(a, ng);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "init launch");
  return ILBM_OK;
}


static int check_box(const ilbm_ctx *ctx, const ilbm_box &b, bool need_out) {
  if (!b.f_in || (need_out && !b.f_out)) {
    set_error("box: f_in/f_out must be set");
    return ILBM_ERR_ARG;
  }
  for (int d = 0; d < ctx->dim; ++d)
    if (b.hi[d] < b.lo[d]) {
      set_error("box: empty valid region");
      return ILBM_ERR_ARG;
    }
  if (b.fstride[0] <= 0 || b.fstride[1] <= 0 || b.fstride[2] <= 0) {
    set_error("box: f strides must be positive");
    return ILBM_ERR_ARG;
  }
  return ILBM_OK;
}

static int check_params(const ilbm_ctx *ctx, const ilbm_level_params *p) {
  if (!p) {
    set_error("level params missing");
    return ILBM_ERR_ARG;
  }
  if (!(p->tau > 0.5)) {
    set_error("tau must exceed 0.5");
    return ILBM_ERR_ARG;
  }
  for (int d = 0; d < ctx->dim; ++d) {
    if (p->periodic[d]) continue;
    for (int s = 0; s < 2; ++s) {
      const int bc = s ? p->bc_hi[d] : p->bc_lo[d];
      if (bc != ILBM_BC_FOEXTRAP && bc != ILBM_BC_EXT_DIR && bc != ILBM_BC_USER_1 &&
          bc != ILBM_BC_USER_2) {
        set_error("non-periodic face needs BC foextrap(2), ext_dir(3), user_1(1001) or user_2(1002)");
        return ILBM_ERR_UNSUPPORTED;
      }
    }
  }
  return ILBM_OK;
}

// Internal entry for the IB: band macro of box `b` into EV (3 x nb) and RHO.
int band_macro(ilbm_ctx *ctx, const ilbm_box &b, const ilbm_level_params *p, const int *blo,
               const int *bn, double *EV, double *RHO, cudaStream_t st) {
  StepArgs a;
  int rc = fill_args(ctx, b, p, a);
  if (rc) return rc;
  return ILBM_DISPATCH(ctx, launch_band_macro, ctx, a, blo, bn, EV, RHO, st);
}

// Band macro on the listed band cells only.
int band_macro_list(ilbm_ctx *ctx, const ilbm_box &b, const ilbm_level_params *p, const int *blo,
                    const int *bn, const int64_t *cells, int ncells, double *EV, double *RHO,
                    cudaStream_t st) {
  StepArgs a;
  int rc = fill_args(ctx, b, p, a);
  if (rc) return rc;
  return ILBM_DISPATCH(ctx, launch_band_macro_list, ctx, a, blo, bn, cells, ncells, EV, RHO, st);
}

// StepArgs of one box of a level, for kernels that take several boxes
int box_step_args(const ilbm_ctx *ctx, const ilbm_box &b, const ilbm_level_params *p,
                  StepArgs *out) {
  return fill_args(ctx, b, p, *out);
}

// Band macro over several boxes whose StepArgs are in device memory.
int band_macro_boxes(ilbm_ctx *ctx, const StepArgs *d_args, int nargs, const int *blo,
                     const int *bn, double *EV, double *RHO, cudaStream_t st) {
  return ILBM_DISPATCH(ctx, launch_band_macro_boxes, ctx, d_args, nargs, blo, bn, EV, RHO, st);
}

// Level step with the band [blo,bhi] deferred until `band_ready`.
int level_step_split(ilbm_ctx *ctx, const ilbm_box &b, const ilbm_level_params *p,
                     const int *blo, const int *bhi, cudaEvent_t band_ready) {
  StepArgs a;
  int rc = fill_args(ctx, b, p, a);
  if (rc) return rc;
  return ILBM_DISPATCH(ctx, launch_step_split, ctx, a, blo, bhi, band_ready);
}

// ---- internal entries of the batch engine (batch.cu) ----------------------

// StepArgs of one batched case: self-filled ghosts, one box equal to the
// domain, distinct f_in / f_out with a ghost layer, macro recovered from f
// (macro_in is not read: the case has taken its first step already).
int batch_case_args(const ilbm_ctx *ctx, const ilbm_box &b, const ilbm_level_params *p,
                    StepArgs *out) {
  int rc = check_params(ctx, p);
  if (rc) return rc;
  if (p->ghost_mode != ILBM_GHOST_SELF) {
    set_error("batched cases use self-filled ghosts (ILBM_GHOST_SELF)");
    return ILBM_ERR_ARG;
  }
  for (int d = 0; d < ctx->dim; ++d)
    if (b.lo[d] != p->domain_lo[d] || b.hi[d] != p->domain_hi[d]) {
      set_error("batched case: the box must equal the domain");
      return ILBM_ERR_ARG;
    }
  if ((rc = check_box(ctx, b, true))) return rc;
  if (b.ngrow_f < 1 || b.f_in == b.f_out) {
    set_error("batched case: f arrays need a ghost layer and f_in != f_out");
    return ILBM_ERR_ARG;
  }
  if ((b.force || b.force_prev) && (b.mstride[0] <= 0 || b.mstride[1] <= 0 || b.mstride[2] <= 0)) {
    set_error("batched case: force strides must be positive");
    return ILBM_ERR_ARG;
  }
  ilbm_box bb = b;
  bb.macro_in = nullptr;
  bb.macro_out = nullptr;
  if ((rc = fill_args(ctx, bb, p, *out))) return rc;
  out->ghost_slices = 0;
  return ILBM_OK;
}

// ghost-push chunks of w threads for one case (each thread takes at most one
// ghost cell per slab); 0 when every face is a self-filled periodic one
int batch_ghost_chunks(const ilbm_ctx *ctx, const StepArgs &a, int w) {
  int64_t maxslab = 0;
  for (int d = 0; d < ctx->dim; ++d) {
    if (a.self_fill && a.periodic[d]) continue;
    int64_t s = 1;
    for (int e = 0; e < ctx->dim; ++e)
      if (e != d) s *= (a.hi[e] - a.lo[e] + 3);
    maxslab = std::max(maxslab, s);
  }
  return (int)((maxslab + w - 1) / w);
}

template <class L, int S>
static int launch_step_batch(ilbm_ctx *ctx, const StepArgs *d_args, const StepTile *d_tiles,
                             int ntiles, int w, int blocks, const int *steps, const int *limit,
                             cudaStream_t st) {
  k_step_batch<L, S><<<blocks, w, 0, st>>>(d_args, d_tiles, ntiles, steps, limit);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "batched level step launch");
  return ILBM_OK;
}

int batch_step_launch(ilbm_ctx *ctx, const StepArgs *d_args, const StepTile *d_tiles, int ntiles,
                      int w, int blocks, const int *steps, const int *limit, cudaStream_t st) {
  if (ntiles <= 0) return ILBM_OK;
  return ILBM_DISPATCH(ctx, launch_step_batch, ctx, d_args, d_tiles, ntiles, w, blocks, steps, limit,
                       st);
}

template <class L, int S>
static int launch_band_macro_batch(ilbm_ctx *ctx, const StepArgs *d_args, const BandDesc *d_bands,
                                   const ItemRef *d_tiles, int ntiles, const int *steps,
                                   const int *limit, cudaStream_t st) {
  const int blocks = std::min(ntiles, 4096);
  k_band_macro_batch<L, S><<<blocks, kItemTile, 0, st>>>(d_args, d_bands, d_tiles, ntiles, steps, limit);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "batched band macro launch");
  return ILBM_OK;
}

int batch_band_macro_launch(ilbm_ctx *ctx, const StepArgs *d_args, const BandDesc *d_bands,
                            const ItemRef *d_tiles, int ntiles, const int *steps, const int *limit,
                            cudaStream_t st) {
  if (ntiles <= 0) return ILBM_OK;
  return ILBM_DISPATCH(ctx, launch_band_macro_batch, ctx, d_args, d_bands, d_tiles, ntiles, steps,
                       limit, st);
}

template <class L, int S>
static int occupancy_step_batch(const ilbm_ctx *, int w, int *per_sm) {
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_step_batch<L, S>, w, 0);
  if (e != cudaSuccess) return cuda_fail(e, "batched level step occupancy");
  return ILBM_OK;
}

// resident blocks of w threads per SM for the batched level step
int batch_step_occupancy(const ilbm_ctx *ctx, int w, int *per_sm) {
  return ILBM_DISPATCH(ctx, occupancy_step_batch, ctx, w, per_sm);
}

// ---- derived fields and refinement tags ------------------------------------
// UpdateDerivedMacroFields / visPara (Source/Core/AmrCoreLBM.cpp:105-168,
// Source/LBM/visPara.H:10-54): vorticity from central differences of the
// FillPatched velocity (2D: dv/dx - du/dy; 3D: |curl u|) and pressure
// (rho - 1)/3 on valid cells; the band macro over the box grown by one gives
// the ghost values with the FillPatch rules.  Also the level maximum of the
// vorticity (ErrorEst's vortMax, AmrCoreLBM.cpp:1047) as block partials.
struct DeriveArgs {
  int dim;
  int lo[3], hi[3];
  int blo[3], bn[3];
  int64_t nb;
  int mgl[3];
  int64_t ms0, ms1;
  double dx[3];
};

__device__ __forceinline__ double ev_at(const DeriveArgs &d, const double *EV, int c, int i, int j, int k) {
  return EV[(int64_t)c * d.nb + (i - d.blo[0]) + (int64_t)(j - d.blo[1]) * d.bn[0] +
            (int64_t)(k - d.blo[2]) * d.bn[0] * d.bn[1]];
}

template <class R>
__global__ void __launch_bounds__(256) k_derive(DeriveArgs d, const double *EV, const double *RHO,
                                                R *vor, R *pres, double *bmax) {
  __shared__ double sh[8];
  const int nx = d.hi[0] - d.lo[0] + 1, ny = d.hi[1] - d.lo[1] + 1;
  const int nz = (d.dim == 3) ? d.hi[2] - d.lo[2] + 1 : 1;
  const int64_t n = (int64_t)nx * ny * nz;
  double mx = -1.0e300;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int i = d.lo[0] + (int)(t % nx), j = d.lo[1] + (int)((t / nx) % ny);
    const int k = (d.dim == 3) ? d.lo[2] + (int)(t / ((int64_t)nx * ny)) : 0;
    const double dv_dx = X::div(X::sub(ev_at(d, EV, 1, i + 1, j, k), ev_at(d, EV, 1, i - 1, j, k)),
                                X::mul(2.0, d.dx[0]));
    const double du_dy = X::div(X::sub(ev_at(d, EV, 0, i, j + 1, k), ev_at(d, EV, 0, i, j - 1, k)),
                                X::mul(2.0, d.dx[1]));
    double w;
    if (d.dim == 3) {
      const double du_dz = X::div(X::sub(ev_at(d, EV, 0, i, j, k + 1), ev_at(d, EV, 0, i, j, k - 1)),
                                  X::mul(2.0, d.dx[2]));
      const double dw_dx = X::div(X::sub(ev_at(d, EV, 2, i + 1, j, k), ev_at(d, EV, 2, i - 1, j, k)),
                                  X::mul(2.0, d.dx[0]));
      const double dv_dz = X::div(X::sub(ev_at(d, EV, 1, i, j, k + 1), ev_at(d, EV, 1, i, j, k - 1)),
                                  X::mul(2.0, d.dx[2]));
      const double dw_dy = X::div(X::sub(ev_at(d, EV, 2, i, j + 1, k), ev_at(d, EV, 2, i, j - 1, k)),
                                  X::mul(2.0, d.dx[1]));
      const double ox = X::sub(dw_dy, dv_dz), oy = X::sub(du_dz, dw_dx), oz = X::sub(dv_dx, du_dy);
      w = __dsqrt_rn(X::add(X::add(X::mul(ox, ox), X::mul(oy, oy)), X::mul(oz, oz)));
    } else {
      w = X::sub(dv_dx, du_dy);
    }
    const int64_t m = (int64_t)(i - d.mgl[0]) + (int64_t)(j - d.mgl[1]) * d.ms0 +
                      (int64_t)(k - d.mgl[2]) * d.ms1;
    const int64_t b = (i - d.blo[0]) + (int64_t)(j - d.blo[1]) * d.bn[0] +
                      (int64_t)(k - d.blo[2]) * d.bn[0] * d.bn[1];
    if (vor) vor[m] = R(w);
    if (pres) pres[m] = R(X::div(X::sub(RHO[b], 1.0), 3.0));
    mx = fmax(mx, w);
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = sh[0];
    for (int w2 = 1; w2 < (int)(blockDim.x >> 5); ++w2) t = fmax(t, sh[w2]);
    bmax[blockIdx.x] = t;
  }
}

__global__ void k_max_final(const double *bmax, int nb, double *out) {
  if (threadIdx.x == 0) {
    double t = -1.0e300;
    for (int b = 0; b < nb; ++b) t = fmax(t, bmax[b]);
    *out = t;
  }
}

// ErrorEst tagging (AmrCoreLBM.cpp:1145-1180, Tagging.H:12-18) on valid
// cells: cleared inside the no-refine x zones, set where |vorticity| >
// threshold or inside the body refinement box; tags[i + nx*(j + ny*k)].
struct TagArgs {
  int dim;
  int lo[3], hi[3];
  int mgl[3];
  int64_t ms0, ms1;
  double threshold;
  int use_box;
  double box_lo[3], box_hi[3];
  double nr_lo, nr_hi;
  double plo[3], phi[3], dx[3];
  int use_ls;                  // level-set band of a cylinder / sphere body
  double ls_c[3], ls_r, ls_band;
};

template <class R>
__global__ void __launch_bounds__(256) k_tags(TagArgs g, const R *vor, unsigned char *tags,
                                              unsigned long long *count) {
  const int nx = g.hi[0] - g.lo[0] + 1, ny = g.hi[1] - g.lo[1] + 1;
  const int nz = (g.dim == 3) ? g.hi[2] - g.lo[2] + 1 : 1;
  const int64_t n = (int64_t)nx * ny * nz;
  unsigned long long mine = 0;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int i = g.lo[0] + (int)(t % nx), j = g.lo[1] + (int)((t / nx) % ny);
    const int k = (g.dim == 3) ? g.lo[2] + (int)(t / ((int64_t)nx * ny)) : 0;
    const double x = X::add(g.plo[0], X::mul(X::add(double(i), 0.5), g.dx[0]));
    unsigned char tag = 0;
    bool blocked = false;
    if (g.nr_lo > 0.0 || g.nr_hi > 0.0)
      blocked = (x <= X::add(g.plo[0], g.nr_lo)) || (x >= X::sub(g.phi[0], g.nr_hi));
    if (!blocked) {
      const int64_t m = (int64_t)(i - g.mgl[0]) + (int64_t)(j - g.mgl[1]) * g.ms0 +
                        (int64_t)(k - g.mgl[2]) * g.ms1;
      if (fabs(double(vor[m])) > g.threshold) tag = 1;
      if (g.use_ls) {
        // signed distance at the cell centre, as LevelSetManager builds it
        const double y = X::add(g.plo[1], X::mul(X::add(double(j), 0.5), g.dx[1]));
        const double ex = X::sub(x, g.ls_c[0]), ey = X::sub(y, g.ls_c[1]);
        double r2 = X::add(X::mul(ex, ex), X::mul(ey, ey));
        if (g.dim == 3) {
          const double z = X::add(g.plo[2], X::mul(X::add(double(k), 0.5), g.dx[2]));
          const double ez = X::sub(z, g.ls_c[2]);
          r2 = X::add(r2, X::mul(ez, ez));
        }
        if (X::sub(__dsqrt_rn(r2), g.ls_r) < g.ls_band) tag = 1;
      }
      if (g.use_box) {
        const double y = X::add(g.plo[1], X::mul(X::add(double(j), 0.5), g.dx[1]));
        const double z = (g.dim == 3) ? X::add(g.plo[2], X::mul(X::add(double(k), 0.5), g.dx[2])) : 0.0;
        if (x >= g.box_lo[0] && x <= g.box_hi[0] && y >= g.box_lo[1] && y <= g.box_hi[1] &&
            z >= g.box_lo[2] && z <= g.box_hi[2])
          tag = 1;
      }
    }
    tags[t] = tag;
    mine += tag;
  }
  for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd(count, mine);
}

// one level step; with mlo / mhi the boxes' macro_in holds stored values
// only on [mlo, mhi] (elsewhere rho, u are recovered from f^n and F^{n-1}),
// and macro_out is written there only.  part (one box only): 0 = the whole
// step; 1 = the ghost-shell push and the cells of the first half of the box
// along its last dimension; 2 = the cells of the second half, then
// macro_out.  Every (cell, direction) slot of f_out is written by exactly one
// cell or ghost push, so the two halves may run at different times
int level_step_impl(ilbm_ctx *ctx, const ilbm_box *boxes, int nbox, const ilbm_level_params *p,
                    const int *mlo, const int *mhi, int part) {
  if (!ctx || !boxes || nbox <= 0 || part < 0 || part > 2 || (part && nbox != 1)) {
    set_error("level step: null argument");
    return ILBM_ERR_ARG;
  }
  int rc = check_params(ctx, p);
  if (rc) return rc;
  for (int n = 0; n < nbox; ++n)
    if (boxes[n].ngrow_f < 1) {
      set_error("f arrays need at least one ghost layer (edge cells push into it as scratch)");
      return ILBM_ERR_ARG;
    }
  if (p->ghost_mode == ILBM_GHOST_SELF) {
    if (nbox != 1) {
      set_error("self-fill ghost mode needs exactly one box covering the domain");
      return ILBM_ERR_ARG;
    }
    for (int d = 0; d < ctx->dim; ++d)
      if (boxes[0].lo[d] != p->domain_lo[d] || boxes[0].hi[d] != p->domain_hi[d]) {
        set_error("self-fill ghost mode: the box must equal the domain");
        return ILBM_ERR_ARG;
      }

  } else if (p->ghost_mode != ILBM_GHOST_CALLER) {
    set_error("unknown ghost mode");
    return ILBM_ERR_ARG;
  }
  for (int n = 0; n < nbox; ++n) {
    const ilbm_box &b = boxes[n];
    if ((rc = check_box(ctx, b, true))) return rc;
    if (p->ghost_mode == ILBM_GHOST_CALLER && b.ngrow_f < 1) {
      set_error("caller ghost mode needs ngrow_f >= 1");
      return ILBM_ERR_ARG;
    }
    if (p->ghost_mode == ILBM_GHOST_CALLER && (b.macro_in || b.force || b.force_prev) &&
        b.ngrow_m < 1) {
      set_error("caller ghost mode reads macro/force ghosts: needs ngrow_m >= 1");
      return ILBM_ERR_ARG;
    }
    if ((b.macro_in || b.macro_out || b.force || b.force_prev) &&
        (b.mstride[0] <= 0 || b.mstride[1] <= 0 || b.mstride[2] <= 0)) {
      set_error("box: macro/force strides must be positive");
      return ILBM_ERR_ARG;
    }
    if (b.f_in == b.f_out) {
      set_error("f_in and f_out must be distinct (two-lattice scheme)");
      return ILBM_ERR_ARG;
    }
    StepArgs a;
    if ((rc = fill_args(ctx, b, p, a))) return rc;
    if (mlo && mhi) {
      a.use_mbox = 1;
      for (int d = 0; d < 3; ++d) {
        a.mblo[d] = (d < ctx->dim) ? mlo[d] : 0;
        a.mbhi[d] = (d < ctx->dim) ? mhi[d] : 0;
      }
    }
    if (part == 0) {
      rc = ILBM_DISPATCH(ctx, launch_step, ctx, a, p);
    } else if (a.hi[ctx->dim - 1] == a.lo[ctx->dim - 1]) {
      // one cell along the split dimension: the first part takes it all
      if (part == 1) rc = ILBM_DISPATCH(ctx, launch_step_part, ctx, a, true);
    } else {
      const int e = ctx->dim - 1;  // split along the last dimension
      const int mid = a.lo[e] + (a.hi[e] - a.lo[e] + 1) / 2 - 1;
      if (part == 1)
        a.rhi[e] = mid;
      else
        a.rlo[e] = mid + 1;
      rc = ILBM_DISPATCH(ctx, launch_step_part, ctx, a, part == 1);
    }
    if (rc) return rc;
    if (part == 1) continue;  // macro_out once both halves have run
    if (b.macro_out) {
      StepArgs am = a;
      am.f_in = b.f_out;
      int rlo[3] = {a.lo[0], a.lo[1], a.lo[2]}, rhi[3] = {a.hi[0], a.hi[1], a.hi[2]};
      if (a.use_mbox)  // stored values are kept on the macro box only
        for (int d = 0; d < ctx->dim; ++d) {
          rlo[d] = std::max(rlo[d], a.mblo[d]);
          rhi[d] = std::min(rhi[d], a.mbhi[d]);
        }
      rc = ILBM_DISPATCH(ctx, launch_macro, ctx, am, rlo, rhi, b.macro_out);
      if (rc) return rc;
    }
  }
  return ILBM_OK;
}

}  // namespace ilbm

using namespace ilbm;

void *ilbm_ctx_scratch(ilbm_ctx *ctx, size_t n) {
  if (ctx->scratch_bytes >= n) return ctx->scratch;
  if (ctx->scratch) cudaFree(ctx->scratch);
  ctx->scratch = nullptr;
  ctx->scratch_bytes = 0;
  if (cudaMalloc(&ctx->scratch, n) != cudaSuccess) return nullptr;
  ctx->scratch_bytes = n;
  return ctx->scratch;
}

cudaError_t ilbm_ctx_malloc(ilbm_ctx *ctx, void **p, size_t bytes) {
  return cudaMallocFromPoolAsync(p, std::max<size_t>(bytes, 1), ctx->pool, ctx->stream);
}

void ilbm_ctx_free(ilbm_ctx *ctx, void *p) {
  if (p) cudaFreeAsync(p, ctx->stream);
}

extern "C" {

const char *ilbm_last_error(void) { return ilbm::get_error(); }

int ilbm_create(const ilbm_lattice *lat, int storage, int device, void *cuda_stream,
                ilbm_ctx **out) {
  if (!lat || !out) {
    set_error("ilbm_create: null argument");
    return ILBM_ERR_ARG;
  }
  *out = nullptr;
  if (storage < ILBM_STORAGE_F64 || storage > ILBM_STORAGE_F16_SCALED) {
    set_error("ilbm_create: unknown storage form");
    return ILBM_ERR_ARG;
  }
  // the lattice must be one of the three deck orderings, with w = wis/wim
  int dim = 0;
  auto match = [&](auto L) -> bool {
    using LL = decltype(L);
    if (lat->q != LL::Q) return false;
    for (int q = 0; q < LL::Q; ++q) {
      if (lat->cx[q] != double(LL::cx(q)) || lat->cy[q] != double(LL::cy(q)) ||
          lat->cz[q] != double(LL::cz(q)))
        return false;
      if (lat->wim[q] == 0.0 || lat->wis[q] / lat->wim[q] != LL::w(q)) return false;
    }
    dim = LL::D;
    return true;
  };
  if (!(match(Lat<9>{}) || match(Lat<19>{}) || match(Lat<27>{}))) {
    set_error("ilbm_create: lattice must be D2Q9, D3Q19 or D3Q27 in the reference deck order");
    return ILBM_ERR_UNSUPPORTED;
  }
  if (lat->dim != 0 && lat->dim != dim) {
    set_error("ilbm_create: lattice dimension mismatch");
    return ILBM_ERR_ARG;
  }
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  auto *c = new ilbm_ctx();
  c->q = lat->q;
  for (int q = 0; q < lat->q; ++q) c->w[q] = lat->wis[q] / lat->wim[q];
  c->dim = dim;
  c->storage = storage;
  c->device = device;
  if (cuda_stream) {
    c->stream = static_cast<cudaStream_t>(cuda_stream);
  } else {
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      delete c;
      return cuda_fail(e, "cudaStreamCreate");
    }
    c->own_stream = true;
  }
  for (int s = 0; s < 16; ++s) {
    e = cudaEventCreate(&c->ev[s]);
    if (e != cudaSuccess) {
      ilbm_destroy(c);
      return cuda_fail(e, "cudaEventCreate");
    }
  }
  {
    // high-priority side stream for the immersed-boundary chain, which then
    // overlaps the collide-stream of the cells outside its band
    int lo_pri = 0, hi_pri = 0;
    cudaDeviceGetStreamPriorityRange(&lo_pri, &hi_pri);
    e = cudaStreamCreateWithPriority(&c->side, cudaStreamNonBlocking, hi_pri);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_rec, cudaEventDisableTiming);
    if (e != cudaSuccess) {
      ilbm_destroy(c);
      return cuda_fail(e, "side stream");
    }
  }
  e = cudaMallocHost(&c->host_pinned, 64 * sizeof(double));
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) {
    cudaMemPoolProps pp = {};
    pp.allocType = cudaMemAllocationTypePinned;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = device;
    e = cudaMemPoolCreate(&c->pool, &pp);
    uint64_t keep = UINT64_MAX;  // never trim at synchronisation points
    if (e == cudaSuccess) e = cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  if (e != cudaSuccess) {
    ilbm_destroy(c);
    return cuda_fail(e, "ilbm_create");
  }
  *out = c;
  return ILBM_OK;
}

int ilbm_destroy(ilbm_ctx *ctx) {
  if (!ctx) return ILBM_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (int s = 0; s < 16; ++s)
    if (ctx->ev[s]) cudaEventDestroy(ctx->ev[s]);
  for (int s = 0; s < ctx->nxev; ++s)
    if (ctx->xev[s]) cudaEventDestroy(ctx->xev[s]);
  delete[] ctx->xev;
  if (ctx->scratch) cudaFree(ctx->scratch);
  if (ctx->host_pinned) cudaFreeHost(ctx->host_pinned);
  if (ctx->side) {
    cudaStreamSynchronize(ctx->side);
    cudaStreamDestroy(ctx->side);
  }
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
  if (ctx->ev_done) cudaEventDestroy(ctx->ev_done);
  if (ctx->ev_rec) cudaEventDestroy(ctx->ev_rec);
  // a pool with allocations outstanding is released once they are freed
  if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return ILBM_OK;
}

int ilbm_sync(ilbm_ctx *ctx) {
  if (!ctx) return ILBM_ERR_ARG;
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "stream synchronize");
  return ILBM_OK;
}

void *ilbm_stream(ilbm_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

}  // extern "C"

// a recorded sequence of the context's launches, instantiated once
struct ilbm_graph {
  cudaGraphExec_t exec = nullptr;
  int64_t kernels = 0;  // kernel nodes: what one replay adds to the launch count
};

extern "C" {

int ilbm_graph_begin(ilbm_ctx *ctx) {
  if (!ctx) return ILBM_ERR_ARG;
  if (ctx->capture_launch0 >= 0) {
    set_error("ilbm_graph_begin: a capture is already open on this context");
    return ILBM_ERR_ARG;
  }
  cudaSetDevice(ctx->device);
  // thread-local: launches other host threads make meanwhile are not recorded
  cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_graph_begin");
  ctx->capture_launch0 = ctx->launches;
  return ILBM_OK;
}

int ilbm_graph_end(ilbm_ctx *ctx, ilbm_graph **out) {
  if (!ctx || !out) return ILBM_ERR_ARG;
  *out = nullptr;
  if (ctx->capture_launch0 < 0) {
    set_error("ilbm_graph_end: no capture open on this context");
    return ILBM_ERR_ARG;
  }
  ctx->launches = ctx->capture_launch0;  // the recorded launches did not run
  ctx->capture_launch0 = -1;
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
  if (e != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return cuda_fail(e != cudaSuccess ? e : cudaErrorStreamCaptureInvalidated, "ilbm_graph_end");
  }
  size_t nn = 0;
  e = cudaGraphGetNodes(g, nullptr, &nn);
  std::vector<cudaGraphNode_t> nodes(nn);
  if (e == cudaSuccess && nn) e = cudaGraphGetNodes(g, nodes.data(), &nn);
  int64_t kernels = 0;
  for (size_t i = 0; e == cudaSuccess && i < nn; ++i) {
    cudaGraphNodeType t;
    e = cudaGraphNodeGetType(nodes[i], &t);
    if (e == cudaSuccess && t == cudaGraphNodeTypeKernel) ++kernels;
  }
  cudaGraphExec_t exec = nullptr;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_graph_end: instantiate");
  ilbm_graph *h = new ilbm_graph;
  h->exec = exec;
  h->kernels = kernels;
  *out = h;
  return ILBM_OK;
}

int ilbm_graph_launch(ilbm_ctx *ctx, const ilbm_graph *g) {
  if (!ctx || !g || !g->exec) return ILBM_ERR_ARG;
  cudaError_t e = cudaGraphLaunch(g->exec, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_graph_launch");
  ctx->launches += g->kernels;
  return ILBM_OK;
}

int ilbm_graph_destroy(ilbm_graph *g) {
  if (!g) return ILBM_OK;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  delete g;
  return ILBM_OK;
}

static cudaEvent_t *event_slot(ilbm_ctx *ctx, int slot) {
  if (slot < 0 || slot >= 16 + 8192) return nullptr;
  if (slot < 16) return &ctx->ev[slot];
  const int x = slot - 16;
  if (x >= ctx->nxev) {
    const int n = std::max(x + 1, std::max(64, 2 * ctx->nxev));
    auto *nv = new cudaEvent_t[n];
    for (int i = 0; i < ctx->nxev; ++i) nv[i] = ctx->xev[i];
    for (int i = ctx->nxev; i < n; ++i) nv[i] = nullptr;
    delete[] ctx->xev;
    ctx->xev = nv;
    ctx->nxev = n;
  }
  if (!ctx->xev[x] && cudaEventCreate(&ctx->xev[x]) != cudaSuccess) return nullptr;
  return &ctx->xev[x];
}

int ilbm_event_record(ilbm_ctx *ctx, int slot) {
  if (!ctx) return ILBM_ERR_ARG;
  cudaEvent_t *ev = event_slot(ctx, slot);
  if (!ev) {
    set_error("event slot out of range (0..8207)");
    return ILBM_ERR_ARG;
  }
  cudaError_t e = cudaEventRecord(*ev, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaEventRecord");
  return ILBM_OK;
}

int ilbm_event_elapsed_ms(ilbm_ctx *ctx, int a, int b, float *ms) {
  if (!ctx || !ms) return ILBM_ERR_ARG;
  cudaEvent_t *ea = event_slot(ctx, a), *eb = event_slot(ctx, b);
  if (!ea || !eb) {
    set_error("event slot out of range");
    return ILBM_ERR_ARG;
  }
  cudaError_t e = cudaEventSynchronize(*eb);
  if (e != cudaSuccess) return cuda_fail(e, "cudaEventSynchronize");
  e = cudaEventElapsedTime(ms, *ea, *eb);
  if (e != cudaSuccess) return cuda_fail(e, "cudaEventElapsedTime");
  return ILBM_OK;
}

int64_t ilbm_kernel_launches(const ilbm_ctx *ctx) { return ctx ? ctx->launches : -1; }

int ilbm_storage_bytes(const ilbm_ctx *ctx, int *sb, int *rb) {
  if (!ctx) return ILBM_ERR_ARG;
  const int s = ctx->storage == ILBM_STORAGE_F64 ? 8 : (ctx->storage == ILBM_STORAGE_F32_SHIFT ? 4 : 2);
  if (sb) *sb = s;
  if (rb) *rb = ctx->storage == ILBM_STORAGE_F64 ? 8 : 4;
  return ILBM_OK;
}

int ilbm_level_step(ilbm_ctx *ctx, const ilbm_box *boxes, int nbox, const ilbm_level_params *p) {
  return level_step_impl(ctx, boxes, nbox, p, nullptr, nullptr, 0);
}

int ilbm_compute_macro(ilbm_ctx *ctx, const ilbm_box *box, const ilbm_level_params *p,
                       const void *f, const void *force, void *macro_out, const int lo[3],
                       const int hi[3]) {
  if (!ctx || !box || !f || !macro_out) {
    set_error("ilbm_compute_macro: null argument");
    return ILBM_ERR_ARG;
  }
  StepArgs a;
  int rc = fill_args(ctx, *box, p, a);
  if (rc) return rc;
  a.f_in = f;
  a.force = force;
  if (!p) {
    for (int d = 0; d < 3; ++d) {
      a.flo[d] = -(1 << 30);
      a.fhi[d] = (1 << 30);
    }
  }
  int rlo[3], rhi[3];
  for (int d = 0; d < 3; ++d) {
    const bool use = d < ctx->dim;
    rlo[d] = use ? std::max(lo ? lo[d] : box->lo[d], box->lo[d]) : 0;
    rhi[d] = use ? std::min(hi ? hi[d] : box->hi[d], box->hi[d]) : 0;
  }
  return ILBM_DISPATCH(ctx, launch_macro, ctx, a, rlo, rhi, macro_out);
}

int ilbm_init_equilibrium(ilbm_ctx *ctx, const ilbm_box *box) {
  if (!ctx || !box || !box->f_in || !box->f_out || !box->macro_in) {
    set_error("ilbm_init_equilibrium: f_in, f_out and macro_in are required");
    return ILBM_ERR_ARG;
  }
  if (box->ngrow_m < box->ngrow_f) {
    set_error("ilbm_init_equilibrium: macro ghost width must cover the f ghost width");
    return ILBM_ERR_ARG;
  }
  StepArgs a;
  int rc = fill_args(ctx, *box, nullptr, a);
  if (rc) return rc;
  return ILBM_DISPATCH(ctx, launch_init, ctx, a, box->ngrow_f);
}


int ilbm_derived_fields(ilbm_ctx *ctx, const ilbm_box *box, const ilbm_level_params *p,
                        const void *f, const void *force_prev, const double dx[3], void *vor,
                        void *pres, double *vort_max) {
  if (!ctx || !box || !p || !f || !dx) {
    set_error("ilbm_derived_fields: null argument");
    return ILBM_ERR_ARG;
  }
  int rc = check_params(ctx, p);
  if (rc) return rc;
  if (p->ghost_mode != ILBM_GHOST_SELF) {
    set_error("ilbm_derived_fields: needs self-filled ghosts (one box equal to the domain)");
    return ILBM_ERR_UNSUPPORTED;
  }
  for (int d = 0; d < ctx->dim; ++d)
    if (box->lo[d] != p->domain_lo[d] || box->hi[d] != p->domain_hi[d]) {
      set_error("ilbm_derived_fields: the box must equal the domain");
      return ILBM_ERR_ARG;
    }
  if ((vor || pres) && (box->mstride[0] <= 0 || box->mstride[1] <= 0)) {
    set_error("ilbm_derived_fields: macro strides must be positive");
    return ILBM_ERR_ARG;
  }
  ilbm_box b = *box;
  b.f_in = const_cast<void *>(f);
  b.f_out = nullptr;
  b.macro_in = nullptr;
  b.force_prev = const_cast<void *>(force_prev);
  DeriveArgs d;
  std::memset(&d, 0, sizeof(d));
  d.dim = ctx->dim;
  int64_t nb = 1, ncell = 1;
  int blo[3] = {0, 0, 0}, bn[3] = {1, 1, 1};
  for (int q = 0; q < 3; ++q) {
    d.lo[q] = (q < ctx->dim) ? box->lo[q] : 0;
    d.hi[q] = (q < ctx->dim) ? box->hi[q] : 0;
    d.mgl[q] = (q < ctx->dim) ? box->lo[q] - box->ngrow_m : 0;
    if (q < ctx->dim) {
      blo[q] = box->lo[q] - 1;
      bn[q] = box->hi[q] - box->lo[q] + 3;
    }
    d.blo[q] = blo[q];
    d.bn[q] = bn[q];
    nb *= bn[q];
    ncell *= (d.hi[q] - d.lo[q] + 1);
  }
  d.nb = nb;
  d.ms0 = box->mstride[0];
  d.ms1 = box->mstride[1];
  for (int q = 0; q < 3; ++q) d.dx[q] = dx[q];  // the level's xCellSize, yCellSize, zCellSize
  const int blocks = (int)std::min<int64_t>((ncell + 255) / 256, 1184);
  double *scr = static_cast<double *>(ilbm_ctx_scratch(ctx, (4 * nb + blocks + 8) * sizeof(double)));
  if (!scr) {
    set_error("ilbm_derived_fields: scratch allocation failed");
    return ILBM_ERR_NOMEM;
  }
  double *EV = scr, *RHO = scr + 3 * nb, *bmax = scr + 4 * nb, *out = bmax + blocks;
  if ((rc = band_macro(ctx, b, p, blo, bn, EV, RHO, ctx->stream))) return rc;
  if (ctx->storage == ILBM_STORAGE_F64)
    k_derive<double><<<blocks, 256, 0, ctx->stream>>>(d, EV, RHO, static_cast<double *>(vor),
                                                      static_cast<double *>(pres), bmax);
  else
    k_derive<float><<<blocks, 256, 0, ctx->stream>>>(d, EV, RHO, static_cast<float *>(vor),
                                                     static_cast<float *>(pres), bmax);
  k_max_final<<<1, 32, 0, ctx->stream>>>(bmax, blocks, out);
  ctx->launches += 2;
  double mx = 0.0;
  cudaMemcpyAsync(&mx, out, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_derived_fields");
  if (vort_max) *vort_max = mx;
  return ILBM_OK;
}

int ilbm_tag_cells(ilbm_ctx *ctx, const ilbm_box *box, const void *vor, double threshold,
                   int use_box, const double box_lo[3], const double box_hi[3],
                   double no_refine_xlo, double no_refine_xhi, const double prob_lo[3],
                   const double prob_hi[3], const double dx[3], const double *levelset,
                   void *tags, int64_t *ntagged) {
  if (!ctx || !box || !vor || !tags || !prob_lo || !prob_hi || !dx || (use_box && (!box_lo || !box_hi))) {
    set_error("ilbm_tag_cells: null argument");
    return ILBM_ERR_ARG;
  }
  TagArgs g;
  std::memset(&g, 0, sizeof(g));
  g.dim = ctx->dim;
  int64_t ncell = 1;
  for (int q = 0; q < 3; ++q) {
    g.lo[q] = (q < ctx->dim) ? box->lo[q] : 0;
    g.hi[q] = (q < ctx->dim) ? box->hi[q] : 0;
    g.mgl[q] = (q < ctx->dim) ? box->lo[q] - box->ngrow_m : 0;
    ncell *= (g.hi[q] - g.lo[q] + 1);
    g.plo[q] = prob_lo[q];
    g.phi[q] = prob_hi[q];
    g.dx[q] = dx[q];
    if (use_box) {
      g.box_lo[q] = box_lo[q];
      g.box_hi[q] = box_hi[q];
    }
  }
  g.ms0 = box->mstride[0];
  g.ms1 = box->mstride[1];
  g.threshold = threshold;
  g.use_box = use_box;
  g.nr_lo = no_refine_xlo;
  g.nr_hi = no_refine_xhi;
  if (levelset) {
    if (!(levelset[4] >= 0.0) || !(levelset[5] > 0.0)) {
      set_error("ilbm_tag_cells: level-set band cells must be >= 0 and dx_min > 0");
      return ILBM_ERR_ARG;
    }
    g.use_ls = 1;
    for (int q = 0; q < 3; ++q) g.ls_c[q] = levelset[q];
    g.ls_r = levelset[3];
    // (n_cells_band + 0.5) * dx_min
    g.ls_band = (std::floor(levelset[4]) + 0.5) * levelset[5];
  }
  unsigned long long *cnt =
      static_cast<unsigned long long *>(ilbm_ctx_scratch(ctx, 8 * sizeof(unsigned long long)));
  if (!cnt) {
    set_error("ilbm_tag_cells: scratch allocation failed");
    return ILBM_ERR_NOMEM;
  }
  cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), ctx->stream);
  const int blocks = (int)std::min<int64_t>((ncell + 255) / 256, 1184);
  if (ctx->storage == ILBM_STORAGE_F64)
    k_tags<double><<<blocks, 256, 0, ctx->stream>>>(g, static_cast<const double *>(vor),
                                                    static_cast<unsigned char *>(tags), cnt);
  else
    k_tags<float><<<blocks, 256, 0, ctx->stream>>>(g, static_cast<const float *>(vor),
                                                   static_cast<unsigned char *>(tags), cnt);
  ctx->launches++;
  unsigned long long h = 0;
  cudaMemcpyAsync(&h, cnt, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_tag_cells");
  if (ntagged) *ntagged = (int64_t)h;
  return ILBM_OK;
}

}  // extern "C"
