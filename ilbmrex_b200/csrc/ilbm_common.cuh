// Shared device-side definitions for the B200 level-step library.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "ilbm_b200.h"

namespace ilbm {

// ---------------------------------------------------------------------------
// Lattices, in the direction order of the reference decks
// (D2Q9: Examples/Cylinder_flow/inputs:35-40, D3Q19: Examples/SquareDuct_flow/
// inputs:36-41, D3Q27: Examples/Sphere_flow/inputs:34-39).  Weights are
// wis/wim evaluated in double, as AmrCoreLBM.cpp:1218-1221 does at run time.
// ---------------------------------------------------------------------------
template <int Q>
struct Lat;

template <>
struct Lat<9> {
  static constexpr int D = 2;
  static constexpr int Q = 9;
  __host__ __device__ static constexpr int cx(int q) {
    constexpr int t[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
    return t[q];
  }
  __host__ __device__ static constexpr int cy(int q) {
    constexpr int t[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
    return t[q];
  }
  __host__ __device__ static constexpr int cz(int) { return 0; }
  __host__ __device__ static constexpr double w(int q) {
    constexpr double t[9] = {4.0 / 9.0,  1.0 / 9.0,  1.0 / 9.0,  1.0 / 9.0, 1.0 / 9.0,
                             1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
    return t[q];
  }
};

template <>
struct Lat<19> {
  static constexpr int D = 3;
  static constexpr int Q = 19;
  __host__ __device__ static constexpr int cx(int q) {
    constexpr int t[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
    return t[q];
  }
  __host__ __device__ static constexpr int cy(int q) {
    constexpr int t[19] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
    return t[q];
  }
  __host__ __device__ static constexpr int cz(int q) {
    constexpr int t[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
    return t[q];
  }
  __host__ __device__ static constexpr double w(int q) {
    return q == 0 ? 12.0 / 36.0 : (q < 7 ? 2.0 / 36.0 : 1.0 / 36.0);
  }
};

template <>
struct Lat<27> {
  static constexpr int D = 3;
  static constexpr int Q = 27;
  __host__ __device__ static constexpr int cx(int q) {
    constexpr int t[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1,
                           -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
    return t[q];
  }
  __host__ __device__ static constexpr int cy(int q) {
    constexpr int t[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1,
                           1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
    return t[q];
  }
  __host__ __device__ static constexpr int cz(int q) {
    constexpr int t[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0,
                           0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};
    return t[q];
  }
  __host__ __device__ static constexpr double w(int q) {
    return q == 0 ? 8.0 / 27.0 : (q < 7 ? 2.0 / 27.0 : (q < 19 ? 1.0 / 54.0 : 1.0 / 216.0));
  }
};

template <class L>
__host__ __device__ constexpr int opposite(int q) {
  for (int p = 0; p < L::Q; ++p)
    if (L::cx(p) == -L::cx(q) && L::cy(p) == -L::cy(q) && L::cz(p) == -L::cz(q)) return p;
  return q;
}

// ---------------------------------------------------------------------------
// FP64 arithmetic in the reference's operation order, with every product and
// sum rounded separately (no contraction into FMA), so the FP64 storage form
// reproduces the reference's results bit for bit.
// ---------------------------------------------------------------------------
struct X {
  __device__ static __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  __device__ static __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  __device__ static __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  __device__ static __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
};

// feqFunction, Source/LBM/feq.H:9-29 (c and w passed as values so the same
// arithmetic serves compile-time and per-lane directions)
template <int D>
__device__ __forceinline__ double feq64v(double cx, double cy, double cz, double wq, double rho,
                                         double u, double v, double w) {
  double eu, uv;
  if (D == 3) {
    eu = X::add(X::add(X::mul(cx, u), X::mul(cy, v)), X::mul(cz, w));
    uv = X::add(X::add(X::mul(u, u), X::mul(v, v)), X::mul(w, w));
  } else {
    eu = X::add(X::mul(cx, u), X::mul(cy, v));
    uv = X::add(X::mul(u, u), X::mul(v, v));
  }
  // wi * rho * (1.0 + 3.0*eu + 4.5*eu*eu - 1.5*uv)
  const double p = X::sub(X::add(X::add(1.0, X::mul(3.0, eu)), X::mul(X::mul(4.5, eu), eu)),
                          X::mul(1.5, uv));
  return X::mul(X::mul(wq, rho), p);
}
template <class L>
__device__ __forceinline__ double feq64(int q, double rho, double u, double v, double w) {
  return feq64v<L::D>(double(L::cx(q)), double(L::cy(q)), double(L::cz(q)), L::w(q), rho, u, v, w);
}

// equilibrium with all three velocity terms (bc_fill.H:189-200,
// AmrCoreLBM.cpp:2146-2158): always 3D sums, even for 2D lattices
__device__ __forceinline__ double feq64_3v(double cx, double cy, double cz, double wq, double rho,
                                           double u, double v, double w) {
  const double eu = X::add(X::add(X::mul(cx, u), X::mul(cy, v)), X::mul(cz, w));
  const double uv = X::add(X::add(X::mul(u, u), X::mul(v, v)), X::mul(w, w));
  const double p = X::sub(X::add(X::add(1.0, X::mul(3.0, eu)), X::mul(X::mul(4.5, eu), eu)),
                          X::mul(1.5, uv));
  return X::mul(X::mul(wq, rho), p);
}
template <class L>
__device__ __forceinline__ double feq64_3(int q, double rho, double u, double v, double w) {
  return feq64_3v(double(L::cx(q)), double(L::cy(q)), double(L::cz(q)), L::w(q), rho, u, v, w);
}

// BGK relaxation of one population plus its Guo increment
// (collide.H:48-55, collide_forced.H:81-108).  has_force is the cell's
// (fx != 0 || fy != 0 || fz != 0) test.
template <int D>
__device__ __forceinline__ double collide64v(double cx, double cy, double cz, double wq, double f,
                                             double feq, double tau, double ux, double uy,
                                             double uz, double fx, double fy, double fz,
                                             bool has_force) {
  double r = X::sub(X::mul(1.0, f), X::div(X::sub(f, feq), tau));
  if (!has_force) return r;
  const double cs2 = 1.0 / 3.0;
  const double fac = X::sub(1.0, X::div(0.5, tau));
  const double eiu = X::add(X::add(X::mul(cx, ux), X::mul(cy, uy)), X::mul(cz, uz));
  const double c4 = X::mul(cs2, cs2);
  const double termx = X::add(X::div(X::sub(cx, ux), cs2), X::mul(X::div(eiu, c4), cx));
  const double termy = X::add(X::div(X::sub(cy, uy), cs2), X::mul(X::div(eiu, c4), cy));
  const double termz =
      (D == 3) ? X::add(X::div(X::sub(cz, uz), cs2), X::mul(X::div(eiu, c4), cz)) : 0.0;
  const double Si = X::mul(X::mul(wq, fac),
                           X::add(X::add(X::mul(termx, fx), X::mul(termy, fy)), X::mul(termz, fz)));
  return X::add(r, Si);
}
template <class L>
__device__ __forceinline__ double collide64_one(int q, double f, double feq, double tau,
                                                double ux, double uy, double uz, double fx,
                                                double fy, double fz, bool has_force) {
  return collide64v<L::D>(double(L::cx(q)), double(L::cy(q)), double(L::cz(q)), L::w(q), f, feq,
                          tau, ux, uy, uz, fx, fy, fz, has_force);
}

// ---------------------------------------------------------------------------
// Storage forms.  load() returns the working value (f for F64, g = f - w for
// the shifted forms); store() converts it back.
// ---------------------------------------------------------------------------
template <int S>
struct Store;

template <>
struct Store<ILBM_STORAGE_F64> {
  using T = double;
  using R = double;
  static constexpr bool shifted = false;
  __device__ static __forceinline__ R load(const T *p, float) { return *p; }
  __device__ static __forceinline__ R cvt(T v, float) { return v; }
  __device__ static __forceinline__ void store(T *p, R v, float) { *p = v; }
};

template <>
struct Store<ILBM_STORAGE_F32_SHIFT> {
  using T = float;
  using R = float;
  static constexpr bool shifted = true;
  __device__ static __forceinline__ R load(const T *p, float) { return __ldg(p); }
  __device__ static __forceinline__ R cvt(T v, float) { return v; }
  __device__ static __forceinline__ void store(T *p, R v, float) { *p = v; }
};

template <>
struct Store<ILBM_STORAGE_F16_SCALED> {
  using T = __half;
  using R = float;
  static constexpr bool shifted = true;
  // s: per-direction factor w_q / scale
  __device__ static __forceinline__ R load(const T *p, float s) { return __half2float(*p) * s; }
  __device__ static __forceinline__ R cvt(T v, float s) { return __half2float(v) * s; }
  __device__ static __forceinline__ void store(T *p, R v, float s) { *p = __float2half_rn(v / s); }
};

// rho, u of a cell from its populations and the previous force
// (calculateMacroForcing.H:155-166, exact order in FP64)
template <class L>
__device__ __forceinline__ void moments64(const double *f, double Fx, double Fy, double Fz,
                                          double &rho, double &u, double &v, double &w) {
  double r = 0.0, m1 = 0.0, m2 = 0.0, m3 = 0.0;
#pragma unroll
  for (int q = 0; q < L::Q; ++q) {
    r = X::add(r, f[q]);
    m1 = X::add(m1, X::mul(double(L::cx(q)), f[q]));
    m2 = X::add(m2, X::mul(double(L::cy(q)), f[q]));
    m3 = X::add(m3, X::mul(double(L::cz(q)), f[q]));
  }
  rho = r;
  u = X::div(X::add(m1, X::mul(0.5, Fx)), r);
  v = X::div(X::add(m2, X::mul(0.5, Fy)), r);
  w = X::div(X::add(m3, X::mul(0.5, Fz)), r);
}

// shifted form (g = f - w): drho = rho - 1.  Every operation is an explicit
// round-to-nearest intrinsic, so the result is the same in every kernel that
// inlines it (no context-dependent contraction into FMA).
template <class L>
__device__ __forceinline__ void moments32(const float *g, float Fx, float Fy, float Fz,
                                          float &drho, float &u, float &v, float &w) {
  float r = 0.f, m1 = 0.f, m2 = 0.f, m3 = 0.f;
#pragma unroll
  for (int q = 0; q < L::Q; ++q) {
    r = __fadd_rn(r, g[q]);
    if (L::cx(q)) m1 = (L::cx(q) > 0) ? __fadd_rn(m1, g[q]) : __fsub_rn(m1, g[q]);
    if (L::cy(q)) m2 = (L::cy(q) > 0) ? __fadd_rn(m2, g[q]) : __fsub_rn(m2, g[q]);
    if (L::cz(q)) m3 = (L::cz(q) > 0) ? __fadd_rn(m3, g[q]) : __fsub_rn(m3, g[q]);
  }
  drho = r;
  const float inv = __fdiv_rn(1.0f, __fadd_rn(1.0f, r));
  u = __fmul_rn(__fmaf_rn(0.5f, Fx, m1), inv);
  v = __fmul_rn(__fmaf_rn(0.5f, Fy, m2), inv);
  w = __fmul_rn(__fmaf_rn(0.5f, Fz, m3), inv);
}

// shifted equilibrium: f_eq - w_q
__device__ __forceinline__ float feqsv(float cx, float cy, float cz, float wq, float drho, float u,
                                       float v, float w) {
  const float cu = cx * u + cy * v + cz * w;
  const float uu = u * u + v * v + w * w;
  const float P = 3.0f * cu + 4.5f * cu * cu - 1.5f * uu;
  return wq * (drho + (1.0f + drho) * P);
}
template <class L>
__device__ __forceinline__ float feqs(int q, float drho, float u, float v, float w) {
  return feqsv(float(L::cx(q)), float(L::cy(q)), float(L::cz(q)), float(L::w(q)), drho, u, v, w);
}

// ---------------------------------------------------------------------------
// FP32 BGK relaxation with the Guo increment in the shifted form
// (collide.H:48-55, collide_forced.H:81-108 in float), arranged so that a
// direction and its opposite share their arithmetic.  Write c_q = s c' with
// c' the member of the pair whose first nonzero component is +1 (s = +-1):
//   om (feq_q - w_q) = om w drho + om w (1 + drho) (4.5 (c'.u)^2 - 1.5 u.u)
//                      + s 3 om w (1 + drho) (c'.u)
//   Guo increment    = w omh (9 (c'.u)(c'.F) - 3 u.F) + s 3 w omh (c'.F)
//   g*_q             = (1 - om) g_q + [the two lines above]
// Both members of a pair evaluate the same expressions on the same inputs
// (products with s are exact sign flips), so the compiler forms them once:
// about two instructions per direction plus four per pair.
// ---------------------------------------------------------------------------
struct Col32 {
  float u, v, w;      // velocity u^n
  float m15uu;        // -1.5 u.u
  float omd, omr;     // om * drho, om * (1 + drho)
  float omm;          // 1 - om
  float omh;          // 1 - 1 / (2 tau)
  float Fx, Fy, Fz;   // F^n
  float m3uF;         // -3 u.F
  bool hf;            // F^n != 0 (the Guo increment is skipped otherwise, collide_forced.H:81-83)
};

template <class L>
__device__ __forceinline__ Col32 col32_setup(float drho, float u, float v, float w, float om,
                                             float omh, float Fx, float Fy, float Fz) {
  Col32 c;
  c.u = u;
  c.v = v;
  c.w = (L::D == 3) ? w : 0.0f;
  c.m15uu = __fmul_rn(-1.5f, __fmaf_rn(c.w, c.w, __fmaf_rn(v, v, __fmul_rn(u, u))));
  c.omd = __fmul_rn(om, drho);
  c.omr = __fmul_rn(om, __fadd_rn(1.0f, drho));
  c.omm = __fsub_rn(1.0f, om);
  c.omh = omh;
  c.Fx = Fx;
  c.Fy = Fy;
  c.Fz = (L::D == 3) ? Fz : 0.0f;
  c.hf = !(Fx == 0.0f && Fy == 0.0f && c.Fz == 0.0f);
  c.m3uF = __fmul_rn(-3.0f, __fmaf_rn(c.w, c.Fz, __fmaf_rn(v, Fy, __fmul_rn(u, Fx))));
  return c;
}

// sign of the first nonzero component of c_q (1 for the rest direction)
template <class L>
__host__ __device__ constexpr int pair_sign(int q) {
  return L::cx(q) != 0 ? L::cx(q) : (L::cy(q) != 0 ? L::cy(q) : (L::cz(q) != 0 ? L::cz(q) : 1));
}

// c'.x for the canonical member of q's pair (compile-time signs, no products)
template <class L>
__device__ __forceinline__ float canon_dot(int q, float x, float y, float z) {
  const int s = pair_sign<L>(q);
  const int a = s * L::cx(q), b = s * L::cy(q), c = s * L::cz(q);
  float r = 0.0f;
  bool first = true;
  if (a != 0) { r = (a > 0) ? x : -x; first = false; }
  if (b != 0) { r = first ? ((b > 0) ? y : -y) : ((b > 0) ? __fadd_rn(r, y) : __fsub_rn(r, y)); first = false; }
  if (c != 0) { r = first ? ((c > 0) ? z : -z) : ((c > 0) ? __fadd_rn(r, z) : __fsub_rn(r, z)); }
  return r;
}

template <class L>
__device__ __forceinline__ float post32(int q, float g, const Col32 &c) {
  const float wq = float(L::w(q));
  const bool rest = (L::cx(q) == 0 && L::cy(q) == 0 && L::cz(q) == 0);
  const float omrw = __fmul_rn(c.omr, wq), omdw = __fmul_rn(c.omd, wq);
  if (rest) {
    float b = __fmaf_rn(omrw, c.m15uu, omdw);
    if (c.hf) b = __fmaf_rn(__fmul_rn(wq, c.omh), c.m3uF, b);
    return __fmaf_rn(c.omm, g, b);
  }
  const float cu = canon_dot<L>(q, c.u, c.v, c.w);
  const float t = __fmaf_rn(__fmul_rn(4.5f, cu), cu, c.m15uu);
  float b = __fmaf_rn(omrw, t, omdw);
  float p = __fmul_rn(__fmul_rn(3.0f, omrw), cu);
  if (c.hf) {
    const float cF = canon_dot<L>(q, c.Fx, c.Fy, c.Fz);
    const float woh = __fmul_rn(wq, c.omh);
    b = __fmaf_rn(woh, __fmaf_rn(__fmul_rn(9.0f, cu), cF, c.m3uF), b);
    p = __fmaf_rn(__fmul_rn(3.0f, woh), cF, p);
  }
  return __fmaf_rn(c.omm, g, (pair_sign<L>(q) > 0) ? __fadd_rn(b, p) : __fsub_rn(b, p));
}

// ---------------------------------------------------------------------------
// Launch helpers
// ---------------------------------------------------------------------------
struct Box3 {
  int lo[3], hi[3];
};

__host__ __device__ __forceinline__ bool in_box(const int *lo, const int *hi, int i, int j,
                                                int k) {
  return i >= lo[0] && i <= hi[0] && j >= lo[1] && j <= hi[1] && k >= lo[2] && k <= hi[2];
}

void set_error(const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);

// calls FN<Lat<Q>, storage>(...) for the context's lattice and storage form
#define ILBM_DISPATCH(ctx, FN, ...)                                                        \
  [&]() -> int {                                                                           \
    switch ((ctx)->q * 4 + (ctx)->storage) {                                               \
      case 9 * 4 + ILBM_STORAGE_F64: return FN<Lat<9>, ILBM_STORAGE_F64>(__VA_ARGS__);     \
      case 9 * 4 + ILBM_STORAGE_F32_SHIFT: return FN<Lat<9>, ILBM_STORAGE_F32_SHIFT>(__VA_ARGS__); \
      case 9 * 4 + ILBM_STORAGE_F16_SCALED: return FN<Lat<9>, ILBM_STORAGE_F16_SCALED>(__VA_ARGS__); \
      case 19 * 4 + ILBM_STORAGE_F64: return FN<Lat<19>, ILBM_STORAGE_F64>(__VA_ARGS__);   \
      case 19 * 4 + ILBM_STORAGE_F32_SHIFT: return FN<Lat<19>, ILBM_STORAGE_F32_SHIFT>(__VA_ARGS__); \
      case 19 * 4 + ILBM_STORAGE_F16_SCALED: return FN<Lat<19>, ILBM_STORAGE_F16_SCALED>(__VA_ARGS__); \
      case 27 * 4 + ILBM_STORAGE_F64: return FN<Lat<27>, ILBM_STORAGE_F64>(__VA_ARGS__);   \
      case 27 * 4 + ILBM_STORAGE_F32_SHIFT: return FN<Lat<27>, ILBM_STORAGE_F32_SHIFT>(__VA_ARGS__); \
      case 27 * 4 + ILBM_STORAGE_F16_SCALED: return FN<Lat<27>, ILBM_STORAGE_F16_SCALED>(__VA_ARGS__); \
      default: set_error("unsupported lattice/storage"); return ILBM_ERR_UNSUPPORTED;      \
    }                                                                                      \
  }()


}  // namespace ilbm

struct ilbm_ctx {
  int q = 0;
  int dim = 0;
  int storage = 0;
  double w[27] = {};  // lattice weights w_q (wis / wim)
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaEvent_t ev[16] = {};
  // extra timing events (slots >= 16), created on first use
  cudaEvent_t *xev = nullptr;
  int nxev = 0;
  int64_t launches = 0;
  int64_t capture_launch0 = -1;  // launch count when a graph capture began (-1: none)
  // reusable scratch (reductions, level box tables)
  void *scratch = nullptr;
  size_t scratch_bytes = 0;
  double *host_pinned = nullptr;
  // side stream (high priority) and fork/join events for the overlapped
  // immersed-boundary chain
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_done = nullptr;
  cudaEvent_t ev_rec = nullptr;  // a force record taken on the side stream is in place
  int sms = 0;
  // the context's own memory pool for stream-ordered allocations (IB arrays,
  // batch tables): freed memory stays in the pool for the next request
  // instead of a device-wide synchronising cudaFree
  cudaMemPool_t pool = nullptr;
};

// grow ctx scratch to at least n bytes (returns nullptr on failure)
void *ilbm_ctx_scratch(ilbm_ctx *ctx, size_t n);
// stream-ordered allocation from the context's pool, on ctx->stream: usable by
// work queued on that stream (or ordered after it by an event) once it returns
cudaError_t ilbm_ctx_malloc(ilbm_ctx *ctx, void **p, size_t bytes);
// stream-ordered free on ctx->stream: after the work queued before it
void ilbm_ctx_free(ilbm_ctx *ctx, void *p);
