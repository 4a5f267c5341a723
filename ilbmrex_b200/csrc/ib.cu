// Marker direct-forcing immersed boundary on the device, FP64.
//
// Follows IBMarkerDF::update_forcing (Source/IBM/IBMarkerDF.cpp:1522-1917):
// per MDF iteration the markers are placed (update_lagrangian_marker,
// :499-609), the Eulerian velocity is interpolated with the 3/4-point Peskin
// kernel over a 5^d stencil (velocity_interpolation_cic, :612-695), the marker
// force is computed explicitly (:741-873) or from the implicit velocity
// correction system A F = (U_d - U)/dt with A = dv*Sx*Sy*Sz + reg*I
// (:1081-1328), spread back (force_spreading_cic, :1331-1512), summed
// (:1781-1819) and applied to the velocity (:1878-1879); the exported force is
// dt*rho*a (:1889-1911).
//
// B200 form: all Eulerian work is restricted to the support band of the body
// (a fixed box around the marker envelope) instead of whole-level MultiFabs.
// The IVC system is solved on the device with Jacobi-preconditioned CG on a
// CSR operator built on the device (the reference factors a dense n x n LU on
// one host core); CG is run to a relative residual of 1e-14.  All kernel
// arithmetic that mirrors the reference uses round-to-nearest intrinsics in
// the reference's operation order.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <cooperative_groups.h>

#include "batch_internal.h"
#include "ilbm_common.cuh"
#include "state_internal.h"

namespace cgrp = cooperative_groups;

namespace ilbm {
int band_macro(ilbm_ctx *ctx, const ilbm_box &b, const ilbm_level_params *p, const int *blo,
               const int *bn, double *EV, double *RHO, cudaStream_t st);
int box_step_args(const ilbm_ctx *ctx, const ilbm_box &b, const ilbm_level_params *p,
                  StepArgs *out);
int band_macro_boxes(ilbm_ctx *ctx, const StepArgs *d_args, int nargs, const int *blo,
                     const int *bn, double *EV, double *RHO, cudaStream_t st);
int band_macro_list(ilbm_ctx *ctx, const ilbm_box &b, const ilbm_level_params *p, const int *blo,
                    const int *bn, const int64_t *cells, int ncells, double *EV, double *RHO,
                    cudaStream_t st);
int level_step_split(ilbm_ctx *ctx, const ilbm_box &b, const ilbm_level_params *p,
                     const int *blo, const int *bhi, cudaEvent_t band_ready);
}

using namespace ilbm;

namespace {

constexpr double kPi = 3.14159265358979323846;

// delta_function, IBMarkerDF.cpp:70-99 (value / h)
__device__ __forceinline__ double delta_fn(double xf, double xp, double h, int type) {
  const double rr = X::div(fabs(X::sub(xf, xp)), h);
  double value = 0.0;
  if (type == 0) {
    if (rr < 1.0)
      value = X::mul(0.125, X::add(X::sub(3.0, X::mul(2.0, rr)),
                                   __dsqrt_rn(X::sub(X::add(1.0, X::mul(4.0, rr)),
                                                     X::mul(X::mul(4.0, rr), rr)))));
    else if (rr < 2.0)
      value = X::mul(0.125, X::sub(X::sub(5.0, X::mul(2.0, rr)),
                                   __dsqrt_rn(X::sub(X::add(-7.0, X::mul(12.0, rr)),
                                                     X::mul(X::mul(4.0, rr), rr)))));
  } else {
    if (rr < 0.5)
      value = X::div(X::add(1.0, __dsqrt_rn(X::sub(1.0, X::mul(X::mul(3.0, rr), rr)))), 3.0);
    else if (rr < 1.5)
      value = X::div(X::sub(X::sub(5.0, X::mul(3.0, rr)),
                            __dsqrt_rn(X::sub(X::add(-2.0, X::mul(6.0, rr)),
                                              X::mul(X::mul(3.0, rr), rr)))),
                     6.0);
  }
  return X::div(value, h);
}

__device__ __forceinline__ double cell_center(double plo, int i, double dx) {
  return X::add(plo, X::mul(X::add(double(i), 0.5), dx));
}
__device__ __forceinline__ int cell_of(double p, double plo, double dx) {
  return (int)floor(X::div(X::sub(p, plo), dx));
}

// overlap_1d, IBMarkerDF.cpp:123-145
__device__ double overlap_1d(double xa, double xb, double h, int kt, double plo, int ilo,
                             int ihi) {
  const int ia = cell_of(xa, plo, h), ib = cell_of(xb, plo, h);
  int lo = max(ia - 2, ib - 2), hi = min(ia + 2, ib + 2);
  lo = max(lo, ilo);
  hi = min(hi, ihi);
  if (lo > hi) return 0.0;
  double sum = 0.0;
  for (int i = lo; i <= hi; ++i) {
    const double xc = cell_center(plo, i, h);
    sum = X::add(sum, X::mul(X::mul(delta_fn(xc, xa, h, kt), delta_fn(xc, xb, h, kt)), h));
  }
  return sum;
}

struct IBArgs {
  int dim, kt, n;
  double plo[3], dx[3];
  int dlo[3], dhi[3];  // domain (cells)
  int periodic[3];
  int blo[3], bn[3];   // band
  int64_t nb;
  double dv, dt, time, wall_tol;
  // geometry / kinematics
  int geometry_type;
  double x0, y0, z0;
  double ub[3], om[3];
  double box_yhi, lid[3];
  double plo_dom[3], phi_dom[3];  // for periodic wrap of positions
  // user-defined kinematics for this call (host-evaluated trig)
  double kc, ks, komega;
  double pivot_x;
  int renorm_interp, renorm_spread;
  double relax, diag_eps;
  int diag;
};

__device__ __forceinline__ int64_t bidx(const IBArgs &a, int i, int j, int k) {
  return (int64_t)(i - a.blo[0]) + (int64_t)(j - a.blo[1]) * a.bn[0] +
         (int64_t)(k - a.blo[2]) * a.bn[0] * a.bn[1];
}
__device__ __forceinline__ bool in_band(const IBArgs &a, int i, int j, int k) {
  return i >= a.blo[0] && i < a.blo[0] + a.bn[0] && j >= a.blo[1] && j < a.blo[1] + a.bn[1] &&
         k >= a.blo[2] && k < a.blo[2] + a.bn[2];
}

// update_lagrangian_marker (user-defined kinematics) + zeroing, :499-609.
// Static geometries keep the positions computed at creation; the
// Redistribute periodic wrap is applied here.
// kc, ks, komega: cos / sin of the pitch angle and its rate at this step
__device__ __forceinline__ void markers_one(const IBArgs &a, double kc, double ks, double komega,
                                            int m, double *xyz, const double *ref, double *tgt,
                                            double *uvw, double *F) {
  if (a.geometry_type == 2) {
    // IBMUserDefinedGeometry.H:144-175
    const double xr = X::sub(ref[m], a.pivot_x), yr = ref[m + a.n], zr = ref[m + 2 * a.n];
    double x = X::sub(X::add(a.x0, X::mul(kc, xr)), X::mul(ks, yr));
    double y = X::add(X::add(a.y0, X::mul(ks, xr)), X::mul(kc, yr));
    double z = X::add(a.z0, zr);
    tgt[m] = X::mul(-komega, X::sub(y, a.y0));
    tgt[m + a.n] = X::mul(komega, X::sub(x, a.x0));
    tgt[m + 2 * a.n] = 0.0;
    double pos[3] = {x, y, z};
    for (int d = 0; d < a.dim; ++d) {
      if (!a.periodic[d]) continue;
      const double L = a.phi_dom[d] - a.plo_dom[d];
      for (int it = 0; it < 4 && pos[d] < a.plo_dom[d]; ++it) pos[d] += L;
      for (int it = 0; it < 4 && pos[d] >= a.phi_dom[d]; ++it) pos[d] -= L;
    }
    xyz[m] = pos[0];
    xyz[m + a.n] = pos[1];
    xyz[m + 2 * a.n] = (a.dim == 3) ? pos[2] : 0.0;
  }
  for (int c = 0; c < 3; ++c) {
    uvw[m + c * a.n] = 0.0;
    F[m + c * a.n] = 0.0;
  }
}

__global__ void k_markers(IBArgs a, double *xyz, const double *ref, double *tgt, double *uvw,
                          double *F) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.n) return;
  markers_one(a, a.kc, a.ks, a.komega, m, xyz, ref, tgt, uvw, F);
}

// velocity_interpolation_cic, :612-695; clip box = domain grown by 2.
// One warp per marker (the batched stages): the 5 kernel weights per
// direction are evaluated once (the reference re-evaluates the same values
// inside its loops) and the 5^d stencil points are spread over the lanes;
// products keep the reference's (tU*tV)*tW order, the sum is a fixed-order
// warp reduction.  With FP64 storage the single-body path sums in the
// reference's own order instead (interp_seq below).
__device__ __forceinline__ void marker_weights(const IBArgs &a, double px, double py, double pz,
                                               int lane, int &i0, int &j0, int &k0,
                                               double &wx, double &wy, double &wz) {
  i0 = cell_of(px, a.plo[0], a.dx[0]);
  j0 = cell_of(py, a.plo[1], a.dx[1]);
  k0 = (a.dim == 3) ? cell_of(pz, a.plo[2], a.dx[2]) : 0;
  const int o = lane % 5 - 2;
  wx = delta_fn(cell_center(a.plo[0], i0 + o, a.dx[0]), px, a.dx[0], a.kt);
  wy = delta_fn(cell_center(a.plo[1], j0 + o, a.dx[1]), py, a.dx[1], a.kt);
  wz = (a.dim == 3) ? delta_fn(cell_center(a.plo[2], k0 + o, a.dx[2]), pz, a.dx[2], a.kt) : 1.0;
}

__device__ __forceinline__ void target_of(const IBArgs &a, int m, const double *xyz,
                                          const double *tgt, double &ux, double &uy,
                                          double &uz);

// A step's kernel-weight table of the markers (the batched stages, and an
// IVC body on the single-case warp-parallel path): marker m's
// weight at offset o - 2 from its cell in direction d is tw[kTabStride m +
// 5 d + o] (1.0 in the third direction of a 2D lattice), its cell tc[m].  The
// interpolation's lanes 0-4 write it; the spreading and the IVC operator
// build of the same step read it instead of evaluating the kernel again, with
// the very values marker_weights / overlap_1d would compute.
constexpr int kTabStride = 16;

// rhs (optional, row stride ld): the IVC right-hand side (U_target - U)/dt of
// the marker, written once here instead of by every block of the solve;
// tw / tc (optional): the weight table above
__device__ __forceinline__ void interp_one(const IBArgs &a, int m, int lane, const double *xyz,
                                           const double *EV, double *uvw, int *status,
                                           const double *tgt, double *rhs, int ld,
                                           double *tw = nullptr, int4 *tc = nullptr) {
  const double px = xyz[m], py = xyz[m + a.n], pz = xyz[m + 2 * a.n];
  const double d = (a.dim == 3) ? X::mul(X::mul(a.dx[0], a.dx[1]), a.dx[2]) : X::mul(a.dx[0], a.dx[1]);
  int i0, j0, k0;
  double wxl, wyl, wzl;
  marker_weights(a, px, py, pz, lane, i0, j0, k0, wxl, wyl, wzl);
  if (tw && lane < 5) {
    double *row = tw + (int64_t)kTabStride * m;
    row[lane] = wxl;
    row[5 + lane] = wyl;
    row[10 + lane] = wzl;
  }
  if (tc && lane == 0) tc[m] = make_int4(i0, j0, k0, 0);
  const int ilo = a.dlo[0] - 2, ihi = a.dhi[0] + 2, jlo = a.dlo[1] - 2, jhi = a.dhi[1] + 2;
  const int klo = (a.dim == 3) ? a.dlo[2] - 2 : 0, khi = (a.dim == 3) ? a.dhi[2] + 2 : 0;
  const int npts = (a.dim == 3) ? 125 : 25;
  double u = 0.0, v = 0.0, w = 0.0, part = 0.0;
  // every lane runs the same number of iterations so the shuffles stay convergent
  const int nit = (npts + 31) / 32;
  for (int it = 0; it < nit; ++it) {
    const int t = lane + 32 * it;
    const int tt = t < npts ? t : 0;
    const int ii = tt / ((a.dim == 3) ? 25 : 5), jj = (tt / ((a.dim == 3) ? 5 : 1)) % 5;
    const int kk = (a.dim == 3) ? tt % 5 : 2;
    const double tU = __shfl_sync(0xffffffffu, wxl, ii, 32);
    const double tV = __shfl_sync(0xffffffffu, wyl, jj, 32);
    const double tW = __shfl_sync(0xffffffffu, wzl, kk, 32);
    if (t >= npts) continue;
    const int ip = i0 + ii - 2, jp = j0 + jj - 2, kp = (a.dim == 3) ? k0 + kk - 2 : 0;
    if (ip < ilo || ip > ihi || jp < jlo || jp > jhi || kp < klo || kp > khi) continue;
    if (!in_band(a, ip, jp, kp)) {
      atomicOr(status, 1);
      continue;
    }
    const double dvl = (a.dim == 3) ? X::mul(X::mul(tU, tV), tW) : X::mul(tU, tV);
    // points outside the kernel's support add signed zeros: skipping their
    // loads leaves every sum bit for bit as it was
    if (dvl == 0.0) continue;
    const int64_t e = bidx(a, ip, jp, kp);
    part = X::add(part, X::mul(dvl, d));
    u = X::add(u, X::mul(X::mul(dvl, EV[e]), d));
    v = X::add(v, X::mul(X::mul(dvl, EV[e + a.nb]), d));
    if (a.dim == 3) w = X::add(w, X::mul(X::mul(dvl, EV[e + 2 * a.nb]), d));
  }
  for (int o = 16; o > 0; o >>= 1) {
    u = X::add(u, __shfl_down_sync(0xffffffffu, u, o));
    v = X::add(v, __shfl_down_sync(0xffffffffu, v, o));
    w = X::add(w, __shfl_down_sync(0xffffffffu, w, o));
    part = X::add(part, __shfl_down_sync(0xffffffffu, part, o));
  }
  if (lane == 0) {
    if (a.renorm_interp && part > 0.0) {
      u = X::div(u, part);
      v = X::div(v, part);
      w = X::div(w, part);
    }
    u = X::add(uvw[m], u);
    v = X::add(uvw[m + a.n], v);
    w = X::add(uvw[m + 2 * a.n], w);
    uvw[m] = u;
    uvw[m + a.n] = v;
    uvw[m + 2 * a.n] = w;
    if (rhs) {
      double Ux, Uy, Uz;
      target_of(a, m, xyz, tgt, Ux, Uy, Uz);
      rhs[m] = X::div(X::sub(Ux, u), a.dt);
      rhs[m + ld] = X::div(X::sub(Uy, v), a.dt);
      rhs[m + 2 * ld] = X::div(X::sub(Uz, w), a.dt);
    }
  }
}


// rigid_target_velocity / box_target_velocity, :147-182
__device__ __forceinline__ void rigid_target(const IBArgs &a, double x, double y, double z,
                                             double &ux, double &uy, double &uz) {
  if (a.geometry_type == 1) {
    ux = uy = uz = 0.0;
    if (fabs(X::sub(y, a.box_yhi)) <= a.wall_tol) {
      ux = a.lid[0];
      uy = a.lid[1];
      uz = a.lid[2];
    }
    return;
  }
  const double rx = X::sub(x, a.x0), ry = X::sub(y, a.y0), rz = X::sub(z, a.z0);
  const double cx = X::sub(X::mul(a.om[1], rz), X::mul(a.om[2], ry));
  const double cy = X::sub(X::mul(a.om[2], rx), X::mul(a.om[0], rz));
  const double cz = X::sub(X::mul(a.om[0], ry), X::mul(a.om[1], rx));
  ux = X::add(a.ub[0], cx);
  uy = X::add(a.ub[1], cy);
  uz = X::add(a.ub[2], cz);
}

__device__ __forceinline__ void target_of(const IBArgs &a, int m, const double *xyz,
                                          const double *tgt, double &ux, double &uy,
                                          double &uz) {
  if (a.geometry_type == 2) {
    ux = tgt[m];
    uy = tgt[m + a.n];
    uz = tgt[m + 2 * a.n];
  } else {
    const double z = (a.dim == 3) ? xyz[m + 2 * a.n] : 0.0;
    rigid_target(a, xyz[m], xyz[m + a.n], z, ux, uy, uz);
  }
}

// compute_lagrangian_force_explicit, :741-873
__device__ __forceinline__ void force_explicit_one(const IBArgs &a, int m, const double *xyz,
                                                   const double *tgt, const double *uvw, double *F) {
  double Ux, Uy, Uz;
  target_of(a, m, xyz, tgt, Ux, Uy, Uz);
  double denom = a.dt;
  if (a.diag) {
    const double px = xyz[m], py = xyz[m + a.n], pz = xyz[m + 2 * a.n];
    const double dV = (a.dim == 3) ? X::mul(X::mul(a.dx[0], a.dx[1]), a.dx[2]) : X::mul(a.dx[0], a.dx[1]);
    const int i0 = cell_of(px, a.plo[0], a.dx[0]), j0 = cell_of(py, a.plo[1], a.dx[1]);
    const int k0 = (a.dim == 3) ? cell_of(pz, a.plo[2], a.dx[2]) : 0;
    double sum2 = 0.0;
    for (int ii = -2; ii < 3; ++ii) {
      const int ip = i0 + ii;
      if (ip < a.dlo[0] || ip > a.dhi[0]) continue;
      const double tU = delta_fn(cell_center(a.plo[0], ip, a.dx[0]), px, a.dx[0], a.kt);
      for (int jj = -2; jj < 3; ++jj) {
        const int jp = j0 + jj;
        if (jp < a.dlo[1] || jp > a.dhi[1]) continue;
        const double tV = delta_fn(cell_center(a.plo[1], jp, a.dx[1]), py, a.dx[1], a.kt);
        if (a.dim == 3) {
          for (int kk = -2; kk < 3; ++kk) {
            const int kp = k0 + kk;
            if (kp < a.dlo[2] || kp > a.dhi[2]) continue;
            const double tW = delta_fn(cell_center(a.plo[2], kp, a.dx[2]), pz, a.dx[2], a.kt);
            const double dvl = X::mul(X::mul(tU, tV), tW);
            sum2 = X::add(sum2, X::mul(X::mul(dvl, dvl), dV));
          }
        } else {
          const double dvl = X::mul(tU, tV);
          sum2 = X::add(sum2, X::mul(X::mul(dvl, dvl), dV));
        }
      }
    }
    const double mkk = X::mul(a.dv, sum2);
    denom = X::mul(a.dt, fmax(mkk, a.diag_eps));
  }
  F[m] = X::add(F[m], X::div(X::mul(a.relax, X::sub(Ux, uvw[m])), denom));
  F[m + a.n] = X::add(F[m + a.n], X::div(X::mul(a.relax, X::sub(Uy, uvw[m + a.n])), denom));
  F[m + 2 * a.n] = X::add(F[m + 2 * a.n], X::div(X::mul(a.relax, X::sub(Uz, uvw[m + 2 * a.n])), denom));
}

__global__ void k_force_explicit(IBArgs a, const double *xyz, const double *tgt,
                                 const double *uvw, double *F) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.n) return;
  force_explicit_one(a, m, xyz, tgt, uvw, F);
}

// ---------------------------------------------------------------------------
// IVC operator (CSR) and Jacobi-preconditioned CG, one CTA per body.
// A_ij = dv * Sx * Sy [* Sz] (+ reg on the diagonal), IBMarkerDF.cpp:1106-1127.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool may_couple(const IBArgs &a, const double *xyz, int i, int j) {
  for (int d = 0; d < a.dim; ++d) {
    const int ci = cell_of(xyz[i + d * a.n], a.plo[d], a.dx[d]);
    const int cj = cell_of(xyz[j + d * a.n], a.plo[d], a.dx[d]);
    if (abs(ci - cj) > 4) return false;
  }
  return true;
}

__device__ double ivc_entry(const IBArgs &a, const double *xyz, int i, int j, double reg) {
  const double sx = overlap_1d(xyz[i], xyz[j], a.dx[0], a.kt, a.plo[0], a.dlo[0], a.dhi[0]);
  const double sy = overlap_1d(xyz[i + a.n], xyz[j + a.n], a.dx[1], a.kt, a.plo[1], a.dlo[1], a.dhi[1]);
  const double sz = (a.dim == 3) ? overlap_1d(xyz[i + 2 * a.n], xyz[j + 2 * a.n], a.dx[2], a.kt,
                                              a.plo[2], a.dlo[2], a.dhi[2])
                                 : 1.0;
  double val = X::mul(X::mul(X::mul(a.dv, sx), sy), sz);
  if (i == j) val = X::add(val, reg);
  return val;
}

// the same coupling test and entry from the step's weight table (kTabStride):
// overlap_1d's nodes, clipping, products and summation order, with the kernel
// values read instead of evaluated
__device__ __forceinline__ int tab_cell(const int4 &c, int d) {
  return d == 0 ? c.x : (d == 1 ? c.y : c.z);
}
__device__ __forceinline__ bool may_couple_tab(const IBArgs &a, const int4 *tc, int i, int j) {
  const int4 ci = tc[i], cj = tc[j];
  return abs(ci.x - cj.x) <= 4 && abs(ci.y - cj.y) <= 4 && (a.dim < 3 || abs(ci.z - cj.z) <= 4);
}
__device__ double ivc_entry_tab(const IBArgs &a, const double *tw, const int4 *tc, int i, int j,
                                double reg) {
  const int4 ci = tc[i], cj = tc[j];
  const double *wi = tw + (int64_t)kTabStride * i, *wj = tw + (int64_t)kTabStride * j;
  auto overlap = [&](int d) {
    const int ia = tab_cell(ci, d), ib = tab_cell(cj, d);
    int lo = max(ia - 2, ib - 2), hi = min(ia + 2, ib + 2);
    lo = max(lo, a.dlo[d]);
    hi = min(hi, a.dhi[d]);
    double sum = 0.0;  // stays 0 when lo > hi, as overlap_1d
    for (int q = lo; q <= hi; ++q)
      sum = X::add(sum, X::mul(X::mul(wi[5 * d + q - ia + 2], wj[5 * d + q - ib + 2]), a.dx[d]));
    return sum;
  };
  const double sx = overlap(0), sy = overlap(1), sz = (a.dim == 3) ? overlap(2) : 1.0;
  double val = X::mul(X::mul(X::mul(a.dv, sx), sy), sz);
  if (i == j) val = X::add(val, reg);
  return val;
}

__device__ double block_sum(double v, double *sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (wid == 0) {
    t = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (lane == 0) sh[32] = t;
  }
  __syncthreads();
  return sh[32];
}

// Solves A x = b for the three force components at once.  rhs: b = (U_d-U)/dt.
// work: 4 vectors of 3n doubles (r, z, p, Ap).  F += x on exit.
// warm: start from the previous solution in X_ (the force changes little
// from one step to the next), else from zero
// fixed-order block reduction of NV values per thread; every thread gets the
// totals in out (sh: kMaxWarps x NV doubles, not shared with a reduction that
// may still be read)
constexpr int kMaxWarps = 32;
constexpr int kCgThreads = 512;  // one-block CG: 128 registers per thread available
template <int NV>
__device__ __forceinline__ void block_reduce(const double *v, double (*sh)[NV], double *out) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < NV; ++c) {
    double x = v[c];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) sh[wid][c] = x;
  }
  __syncthreads();
  const int nw = (int)(blockDim.x >> 5);
#pragma unroll
  for (int c = 0; c < NV; ++c) {
    double t = 0.0;
    for (int w = 0; w < nw; ++w) t += sh[w][c];
    out[c] = t;
  }
}

// One CSR row times three vectors (entries j, j + n, j + 2n of v3), one
// thread: the index and value loads of four entries are issued before their
// gathers, and the gathers before the multiply-adds, which run in entry
// order as the straight loop's do (same partial sums, fewer dependent
// round trips per row).
__device__ __forceinline__ void thread_row_dot3(const int *col, const double *val, int e0, int e1,
                                                const double *v3, int n, double (&acc)[3]) {
  for (int e = e0; e < e1; e += 4) {
    int j[4];
    double v[4], q[4][3];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      j[u] = (e + u < e1) ? col[e + u] : 0;
      v[u] = (e + u < e1) ? val[e + u] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (e + u < e1) {
        q[u][0] = v3[j[u]];
        q[u][1] = v3[j[u] + n];
        q[u][2] = v3[j[u] + 2 * n];
      }
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (e + u < e1) {
        acc[0] += v[u] * q[u][0];
        acc[1] += v[u] * q[u][1];
        acc[2] += v[u] * q[u][2];
      }
  }
}

// systems up to this size keep the search direction in shared memory (p_sh,
// 3 kCgSharedN doubles of the calling kernel)
constexpr int kCgSharedN = 1024;

// Jacobi-preconditioned CG for the three force components at once, one
// block.  warm: start from the previous solution in X_ (the force changes
// little from one step to the next), else from zero.  Per iteration two
// fused reductions (p.Ap; r.z and r.r) keep the block barriers to five.
// hist: the solutions the start may use (0: none, 1: X, 2: X and Xh), kept
// on the device so that the batched solves and the body's own alternate
// freely; x0 = 0, X, or the extrapolation 2 X - Xh
__device__ __forceinline__ void ivc_cg_block(const IBArgs &a, const double *xyz, const double *tgt,
                                             const double *uvw, const int *rowptr, const int *col,
                                             const double *val, const double *diag, double *X_,
                                             double *Xh, int *hist, double *work, double *F,
                                             int maxit, double tol, int *status, int *iters,
                                             double *p_sh) {
  __shared__ double sh3[kMaxWarps][3], sh6[kMaxWarps][6];
  __shared__ int sh_hist;
  const int n = a.n;
  double *r = work, *z = work + 3 * n, *Ap = work + 9 * n;
  double *p = (n <= kCgSharedN) ? p_sh : work + 6 * n;
  if (threadIdx.x == 0) sh_hist = *hist;
  __syncthreads();
  const int h = sh_hist;
  const int warm = h < 2 ? h : 2;
  // b (kept in Ap until the residual is formed), x0
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double Ux, Uy, Uz;
    target_of(a, i, xyz, tgt, Ux, Uy, Uz);
    const double U[3] = {Ux, Uy, Uz};
    for (int c = 0; c < 3; ++c) {
      Ap[i + c * n] = X::div(X::sub(U[c], uvw[i + c * n]), a.dt);
      const double xc = X_[i + c * n];
      if (warm >= 2) X_[i + c * n] = X::sub(X::mul(2.0, xc), Xh[i + c * n]);
      else if (!warm) X_[i + c * n] = 0.0;
      if (warm) Xh[i + c * n] = xc;
    }
  }
  __syncthreads();
  // r = b - A x0, z = r / diag, p = z; partial r.z and b.b
  double part[6] = {0, 0, 0, 0, 0, 0};
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double ax[3] = {0.0, 0.0, 0.0};
    if (warm) thread_row_dot3(col, val, rowptr[i], rowptr[i + 1], X_, n, ax);
    for (int c = 0; c < 3; ++c) {
      const double b = Ap[i + c * n];
      const double rr = b - ax[c];
      r[i + c * n] = rr;
      const double zz = rr / diag[i];
      z[i + c * n] = zz;
      p[i + c * n] = zz;
      part[c] += rr * zz;
      part[3 + c] += b * b;
    }
  }
  double tot[6];
  block_reduce<6>(part, sh6, tot);
  double rz[3] = {tot[0], tot[1], tot[2]};
  const double bn[3] = {sqrt(tot[3]), sqrt(tot[4]), sqrt(tot[5])};
  __syncthreads();  // sh6 is read before the loop reuses it, Ap before it is overwritten
  int it = 0;
  bool done = false;
  for (; it < maxit; ++it) {
    // Ap = A p with the partial p.Ap
    double pap[3] = {0.0, 0.0, 0.0};
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      double acc[3] = {0.0, 0.0, 0.0};
      thread_row_dot3(col, val, rowptr[i], rowptr[i + 1], p, n, acc);
      for (int c = 0; c < 3; ++c) {
        Ap[i + c * n] = acc[c];
        pap[c] += p[i + c * n] * acc[c];
      }
    }
    double pt[3];
    block_reduce<3>(pap, sh3, pt);
    double alpha[3];
    for (int c = 0; c < 3; ++c) alpha[c] = (pt[c] != 0.0) ? rz[c] / pt[c] : 0.0;
    // x += alpha p, r -= alpha Ap, z = r / diag with the partial r.z, r.r
    double q6[6] = {0, 0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < n; i += blockDim.x)
      for (int c = 0; c < 3; ++c) {
        X_[i + c * n] += alpha[c] * p[i + c * n];
        const double rr = r[i + c * n] - alpha[c] * Ap[i + c * n];
        r[i + c * n] = rr;
        const double zz = rr / diag[i];
        z[i + c * n] = zz;
        q6[c] += rr * zz;
        q6[3 + c] += rr * rr;
      }
    double qt[6];
    block_reduce<6>(q6, sh6, qt);
    double beta[3];
    bool ok = true;
    for (int c = 0; c < 3; ++c) {
      beta[c] = (rz[c] != 0.0) ? qt[c] / rz[c] : 0.0;
      rz[c] = qt[c];
      ok = ok && (sqrt(qt[3 + c]) <= tol * bn[c]);
    }
    if (ok) {  // every thread holds the same totals: a uniform exit
      done = true;
      ++it;
      break;
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x)
      for (int c = 0; c < 3; ++c) p[i + c * n] = z[i + c * n] + beta[c] * p[i + c * n];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    *iters = it;
    if (!done) atomicOr(status, 4);
    *hist = (h + 1 < 2) ? h + 1 : 2;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    for (int c = 0; c < 3; ++c) F[i + c * n] = X::add(F[i + c * n], X_[i + c * n]);
}

__global__ void __launch_bounds__(kCgThreads) k_ivc_cg(IBArgs a, const double *xyz, const double *tgt,
                                                 const double *uvw, const int *rowptr,
                                                 const int *col, const double *val,
                                                 const double *diag, double *X_, double *Xh,
                                                 int *hist, double *work, double *F, int maxit,
                                                 double tol, int *status, int *iters) {
  __shared__ double p_sh[3 * kCgSharedN];
  ivc_cg_block(a, xyz, tgt, uvw, rowptr, col, val, diag, X_, Xh, hist, work, F, maxit, tol, status,
               iters, p_sh);
}

// ---------------------------------------------------------------------------
// Multi-CTA CSR build (warp per row) and grid-wide CG for large marker sets
// ---------------------------------------------------------------------------
// tc / tw (optional): the step's weight table, read instead of the positions
__device__ __forceinline__ void csr_count_row(const IBArgs &a, const double *xyz, int *rowptr, int i,
                                              int lane, const int4 *tc = nullptr) {
  int c = 0;
  if (tc)
    for (int j = lane; j < a.n; j += 32) c += may_couple_tab(a, tc, i, j) ? 1 : 0;
  else
    for (int j = lane; j < a.n; j += 32) c += may_couple(a, xyz, i, j) ? 1 : 0;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if (lane == 0) rowptr[i + 1] = c;
}

__global__ void __launch_bounds__(256) k_csr_count(IBArgs a, const double *xyz, int *rowptr,
                                                   const int4 *tc) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < a.n; i += nw)
    csr_count_row(a, xyz, rowptr, i, lane, tc);
}

// exclusive scan of the row counts; if the total exceeds the capacity the
// operator is left empty (every row pointer 0) and status bit 2 is set, so no
// later kernel indexes past the column / value arrays
__device__ __forceinline__ void csr_scan_block(int n, int *rowptr, int cap, int *status) {
  __shared__ int warp_tot[32];
  const int chunk = (n + blockDim.x - 1) / blockDim.x;
  const int s0 = threadIdx.x * chunk, s1 = min(n, s0 + chunk);
  int local = 0;
  for (int i = s0; i < s1; ++i) local += rowptr[i + 1];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = local;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int t = (lane < (int)(blockDim.x >> 5)) ? warp_tot[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    warp_tot[lane] = t;
  }
  __syncthreads();
  int excl = x - local + (wid > 0 ? warp_tot[wid - 1] : 0);
  for (int i = s0; i < s1; ++i) {
    const int c = rowptr[i + 1];
    rowptr[i + 1] = excl + c;
    excl += c;
  }
  if (threadIdx.x == 0) rowptr[0] = 0;
  __syncthreads();
  const int total = rowptr[n];
  __syncthreads();
  if (total > cap) {
    for (int i = s0; i < s1; ++i) rowptr[i + 1] = 0;
    if (threadIdx.x == 0) atomicOr(status, 2);
  }
}

__global__ void __launch_bounds__(1024) k_csr_scan(int n, int *rowptr, int cap, int *status) {
  csr_scan_block(n, rowptr, cap, status);
}

__device__ __forceinline__ void csr_fill_row(const IBArgs &a, const double *xyz, double reg,
                                             const int *rowptr, int *col, double *val,
                                             double *diag, int i, int lane,
                                             const double *tw = nullptr, const int4 *tc = nullptr) {
  {
    int p = rowptr[i];
    for (int j0 = 0; j0 < a.n; j0 += 32) {
      const int j = j0 + lane;
      const bool c = (j < a.n) && (tc ? may_couple_tab(a, tc, i, j) : may_couple(a, xyz, i, j));
      const unsigned m = __ballot_sync(0xffffffffu, c);
      if (c) {
        const int slot = p + __popc(m & ((1u << lane) - 1u));
        const double v = tc ? ivc_entry_tab(a, tw, tc, i, j, reg) : ivc_entry(a, xyz, i, j, reg);
        col[slot] = j;
        val[slot] = v;
        if (i == j) diag[i] = v;
      }
      p += __popc(m);
    }
  }
}

// tw / tc: the step's weight table when the interpolation wrote one, else null
__global__ void __launch_bounds__(256) k_csr_fill(IBArgs a, const double *xyz, double reg,
                                                  const int *rowptr, int *col, double *val,
                                                  double *diag, int cap, int *status,
                                                  const double *tw, const int4 *tc) {
  if ((*status & 2) || rowptr[a.n] > cap) return;  // capacity exceeded (k_csr_scan)
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < a.n; i += nw)
    csr_fill_row(a, xyz, reg, rowptr, col, val, diag, i, lane, tw, tc);
}

// fixed-order reduction of per-block partials (nb blocks x 8 slots); every
// block computes the same values, so branches on them stay grid-uniform
__device__ __forceinline__ void reduce_partials(const double *partial, int nblocks, int nval,
                                                double *out_sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (wid < nval) {
    // eight loads in flight per lane before the adds, which keep the order
    // b = lane, lane + 32, ... (one L2 round trip per eight partials)
    double s = 0.0;
    for (int b0 = lane; b0 < nblocks; b0 += 256) {
      double t[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) t[u] = (b0 + 32 * u < nblocks) ? partial[(b0 + 32 * u) * 8 + wid] : 0.0;
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (b0 + 32 * u < nblocks) s += t[u];
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) out_sh[wid] = s;
  }
  __syncthreads();
}

// block-wide fixed-order sum of nval per-thread values into partial[blockIdx.x*8+c]
__device__ __forceinline__ void block_partials(const double *v, int nval, double (*sh)[8],
                                               double *partial) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int c = 0; c < nval; ++c) {
    double x = v[c];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) sh[wid][c] = x;
  }
  __syncthreads();
  if (threadIdx.x < nval) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w][threadIdx.x];
    partial[blockIdx.x * 8 + threadIdx.x] = t;
  }
  __syncthreads();
}

// Grid-wide preconditioned CG (Jacobi) for the three right-hand sides of the
// IVC system, one cooperative launch.  Two grid barriers per iteration: the
// search direction p = z + beta p_old is formed on the fly by every row that
// reads it (z and p_old are frozen between barriers), the owner storing it in
// the other of two p buffers; block partial sums alternate between two
// buffers, so a block that runs ahead never overwrites partials another
// block is still reducing.  Start: x0 = 0 (warm 0), the previous solution
// (warm 1), or its linear extrapolation 2 x_n - x_{n-1} from the last two
// solutions (warm 2; Xh keeps the history).
// (64 registers: the two resident blocks per SM leave half the register file
// to the level step that runs beside the solve; 96 registers left it one
// block per SM, 0.782-0.788 against 0.762-0.771 ms per coarse step of the
// two-level sphere)
// the solve itself, run by every block of a cooperative grid (sh, red: the
// block's reduction scratch in shared memory)
__device__ __forceinline__ void cg_grid_body(cgrp::grid_group &grid, const IBArgs &a,
                                             const double *xyz, const double *tgt,
                                             const double *uvw, const int *rowptr,
                                             const int *col, const double *val,
                                             const double *diag, double *X_, double *Xh,
                                             double *work, double *F, double *partial, int maxit,
                                             double tol, int *hist, int *status, int *iters,
                                             double (*sh)[8], double *red) {
  const int n = a.n;
  // the start (hist, as the block solve keeps it): read by every block before
  // the first grid barrier, advanced by one thread after the last
  const int h = *hist;
  const int warm = h < 2 ? h : 2;
  double *r = work, *z = work + 3 * n, *Ap = work + 9 * n;
  double *P[2] = {work + 6 * n, work + 12 * n};
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gsz = gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31, nw = gsz >> 5, gw = gtid >> 5;
  double *pbuf[2] = {partial, partial + 8 * gridDim.x};
  int k = 0;  // reductions so far (selects the partials buffer)
  if (warm >= 2) {
    for (int i = gtid; i < 3 * n; i += gsz) {
      const double xc = X_[i];
      X_[i] = X::sub(X::mul(2.0, xc), Xh[i]);
      Xh[i] = xc;
    }
    grid.sync();
  } else if (warm == 1) {
    for (int i = gtid; i < 3 * n; i += gsz) Xh[i] = X_[i];
  }
  // r0 = b - A x0, z0 = r0 / diag; one warp per row
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int row = gw; row < n; row += nw) {
    double s0 = 0, s1 = 0, s2 = 0;
    if (warm) {
      for (int e = rowptr[row] + lane; e < rowptr[row + 1]; e += 32) {
        const double v = val[e];
        const int j = col[e];
        s0 += v * X_[j];
        s1 += v * X_[j + n];
        s2 += v * X_[j + 2 * n];
      }
      for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
      }
    }
    if (lane == 0) {
      double Ux, Uy, Uz;
      target_of(a, row, xyz, tgt, Ux, Uy, Uz);
      const double U[3] = {Ux, Uy, Uz};
      const double ax[3] = {s0, s1, s2};
      for (int c = 0; c < 3; ++c) {
        const double b = X::div(X::sub(U[c], uvw[row + c * n]), a.dt);
        if (!warm) X_[row + c * n] = 0.0;
        const double rr = b - ax[c];
        const double zz = rr / diag[row];
        r[row + c * n] = rr;
        z[row + c * n] = zz;
        acc[c] += rr * zz;
        acc[3 + c] += b * b;
      }
    }
  }
  block_partials(acc, 6, sh, pbuf[k & 1]);
  grid.sync();
  reduce_partials(pbuf[k & 1], gridDim.x, 6, red);
  ++k;
  double rz[3] = {red[0], red[1], red[2]};
  const double bn[3] = {sqrt(red[3]), sqrt(red[4]), sqrt(red[5])};
  double beta[3] = {0.0, 0.0, 0.0};
  __syncthreads();
  int it = 0, cur = 0;  // P[cur]: the previous search direction
  bool done = false;
  for (; it < maxit; ++it) {
    double *pold = P[cur], *pnew = P[cur ^ 1];
    // p = z + beta p_old, formed by every reader; Ap = A p; partial p.Ap
    // (lane c < 3 owns component c of the row: its p entries are loaded
    // before the row's products)
    double pap_c = 0.0;
    const double beta_c = (lane == 0) ? beta[0] : ((lane == 1) ? beta[1] : beta[2]);
    // a warp takes its rows two at a time (row and row + nw) with separate
    // sums, so that the loads of both are in flight together; each row's sum
    // and the order of the rows' p.Ap contributions are those of one row at
    // a time
    for (int row = gw; row < n; row += 2 * nw) {
      const int rb = row + nw;
      const bool two = rb < n;
      double zc = 0.0, pc = 0.0, zb = 0.0, pb = 0.0;
      if (lane < 3) {
        zc = z[row + lane * n];
        if (it) pc = pold[row + lane * n];
        if (two) {
          zb = z[rb + lane * n];
          if (it) pb = pold[rb + lane * n];
        }
      }
      const int ea1 = rowptr[row + 1];
      const int eb0 = two ? rowptr[rb] : 0, eb1 = two ? rowptr[rb + 1] : 0;
      double s0 = 0, s1 = 0, s2 = 0, t0 = 0, t1 = 0, t2 = 0;
      for (int ea = rowptr[row] + lane, eb = eb0 + lane; ea < ea1 || eb < eb1; ea += 32, eb += 32) {
        if (ea < ea1) {
          const double v = val[ea];
          const int j = col[ea];
          const double p0 = it ? __fma_rn(beta[0], pold[j], z[j]) : z[j];
          const double p1 = it ? __fma_rn(beta[1], pold[j + n], z[j + n]) : z[j + n];
          const double p2 = it ? __fma_rn(beta[2], pold[j + 2 * n], z[j + 2 * n]) : z[j + 2 * n];
          s0 += v * p0;
          s1 += v * p1;
          s2 += v * p2;
        }
        if (eb < eb1) {
          const double v = val[eb];
          const int j = col[eb];
          const double p0 = it ? __fma_rn(beta[0], pold[j], z[j]) : z[j];
          const double p1 = it ? __fma_rn(beta[1], pold[j + n], z[j + n]) : z[j + n];
          const double p2 = it ? __fma_rn(beta[2], pold[j + 2 * n], z[j + 2 * n]) : z[j + 2 * n];
          t0 += v * p0;
          t1 += v * p1;
          t2 += v * p2;
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
        t0 += __shfl_xor_sync(0xffffffffu, t0, o);
        t1 += __shfl_xor_sync(0xffffffffu, t1, o);
        t2 += __shfl_xor_sync(0xffffffffu, t2, o);
      }
      if (lane < 3) {
        const int ii = row + lane * n;
        const double sc = (lane == 0) ? s0 : ((lane == 1) ? s1 : s2);
        const double pv = it ? __fma_rn(beta_c, pc, zc) : zc;
        pnew[ii] = pv;
        Ap[ii] = sc;
        pap_c += pv * sc;
        if (two) {
          const int ib = rb + lane * n;
          const double sb = (lane == 0) ? t0 : ((lane == 1) ? t1 : t2);
          const double pvb = it ? __fma_rn(beta_c, pb, zb) : zb;
          pnew[ib] = pvb;
          Ap[ib] = sb;
          pap_c += pvb * sb;
        }
      }
    }
    double pap[3];
    for (int c = 0; c < 3; ++c) pap[c] = (lane == c) ? pap_c : 0.0;
    block_partials(pap, 3, sh, pbuf[k & 1]);
    grid.sync();
    reduce_partials(pbuf[k & 1], gridDim.x, 3, red);
    ++k;
    double alpha[3];
    for (int c = 0; c < 3; ++c) alpha[c] = (red[c] != 0.0) ? rz[c] / red[c] : 0.0;
    __syncthreads();
    double ac[6] = {0, 0, 0, 0, 0, 0};
    for (int i = gtid; i < n; i += gsz)
      for (int c = 0; c < 3; ++c) {
        X_[i + c * n] += alpha[c] * pnew[i + c * n];
        const double rr = r[i + c * n] - alpha[c] * Ap[i + c * n];
        r[i + c * n] = rr;
        const double zz = rr / diag[i];
        z[i + c * n] = zz;
        ac[c] += rr * zz;
        ac[3 + c] += rr * rr;
      }
    block_partials(ac, 6, sh, pbuf[k & 1]);
    grid.sync();
    reduce_partials(pbuf[k & 1], gridDim.x, 6, red);
    ++k;
    bool ok = true;
    for (int c = 0; c < 3; ++c) {
      beta[c] = (rz[c] != 0.0) ? red[c] / rz[c] : 0.0;
      rz[c] = red[c];
      ok = ok && (sqrt(red[3 + c]) <= tol * bn[c]);
    }
    __syncthreads();
    cur ^= 1;
    if (ok) {
      done = true;
      ++it;
      break;
    }
  }
  if (gtid == 0) {
    *iters = it;
    if (!done) atomicOr(status, 4);
    *hist = (h + 1 < 2) ? h + 1 : 2;
  }
  for (int i = gtid; i < n; i += gsz)
    for (int c = 0; c < 3; ++c) F[i + c * n] = X::add(F[i + c * n], X_[i + c * n]);
}

__global__ void __launch_bounds__(256, 4) k_ivc_cg_grid(IBArgs a, const double *xyz, const double *tgt,
                                                     const double *uvw, const int *rowptr,
                                                     const int *col, const double *val,
                                                     const double *diag, double *X_, double *Xh,
                                                     double *work, double *F, double *partial,
                                                     int maxit, double tol, int *hist, int *status,
                                                     int *iters) {
  cgrp::grid_group grid = cgrp::this_grid();
  __shared__ double sh[8][8];
  __shared__ double red[8];
  cg_grid_body(grid, a, xyz, tgt, uvw, rowptr, col, val, diag, X_, Xh, work, F, partial, maxit, tol,
               hist, status, iters, sh, red);
}

// ---------------------------------------------------------------------------
// Fixed IVC operator: explicit inverse and one dense solve per step
// ---------------------------------------------------------------------------
// When the markers do not move and the matrix is not rebuilt, the reference
// factorises A = dv*S*S^T + reg*I once (dense LU, IBMarkerDF.cpp) and
// back-substitutes every step.  Triangular solves are a chain of n dependent
// steps; on the GPU the same once-per-body work is better spent forming A^-1
// (in-place Gauss-Jordan, no pivoting: A is symmetric positive definite), so
// that each step's solve is one bandwidth-bound matvec with three right-hand
// sides and no grid-wide synchronisation.

// CSR -> dense rows (row stride ld, padding columns stay zero)
__global__ void __launch_bounds__(256) k_dense_scatter(int n, int ld, const int *rowptr,
                                                       const int *col, const double *val,
                                                       double *M) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw)
    for (int e = rowptr[i] + lane; e < rowptr[i + 1]; e += 32) M[(size_t)i * ld + col[e]] = val[e];
}

// Gauss-Jordan step k, part 1: pivot row scaled by 1/p, pivot column saved
__global__ void __launch_bounds__(256) k_gj_panel(double *M, int n, int ld, int k, double *rowk,
                                                  double *colk, int *status) {
  const double piv = M[(size_t)k * ld + k];
  if (!(piv > 0.0)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(status + 1, 8);
    return;
  }
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    rowk[t] = (t == k) ? 1.0 / piv : M[(size_t)k * ld + t] / piv;
    colk[t] = M[(size_t)t * ld + k];
  }
}

// part 2, one row per block: a_ij -= a_ik * a_kj/p, a_ik = -a_ik/p, row k = row k/p
__global__ void __launch_bounds__(256) k_gj_update(double *M, int n, int ld, int k,
                                                   const double *rowk, const double *colk,
                                                   const int *status) {
  if (status[1] & 8) return;
  const int i = blockIdx.x;
  double *Mi = M + (size_t)i * ld;
  if (i == k) {
    for (int j = threadIdx.x; j < n; j += blockDim.x) Mi[j] = rowk[j];
    return;
  }
  const double ci = colk[i];
  if (ci == 0.0) return;  // rows not yet coupled to k are unchanged (a_ik stays 0)
  const double rkk = rowk[k];
  for (int j = threadIdx.x; j < n; j += blockDim.x)
    Mi[j] = (j == k) ? -ci * rkk : Mi[j] - ci * rowk[j];
}

// F += A^-1 b with b = (U_target - U_interp)/dt (the IVC right-hand side of
// IBMarkerDF.cpp's solve, written by k_interp with row stride ld, padding
// zero).  One block per row: the 256 threads issue all their loads of the row
// at once (coalesced, up to 8 x 16 bytes each), b comes through L1, and a
// fixed-order block reduction gives the three components.
constexpr int kDenseThreads = 256;
__device__ __forceinline__ void dense_row(const IBArgs &a, const double *rhs, const double *Ainv,
                                          int ld, double *F, int row) {
  __shared__ double red[kDenseThreads / 32][3];
  const int n = a.n;
  const int half = ld >> 1;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const double2 *Ar = reinterpret_cast<const double2 *>(Ainv + (size_t)row * ld);
  const double2 *b0 = reinterpret_cast<const double2 *>(rhs);
  const double2 *b1 = reinterpret_cast<const double2 *>(rhs + ld);
  const double2 *b2 = reinterpret_cast<const double2 *>(rhs + 2 * ld);
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll 8
  for (int h = threadIdx.x; h < half; h += kDenseThreads) {
    const double2 v = __ldcs(Ar + h);
    const double2 x0 = __ldg(b0 + h), x1 = __ldg(b1 + h), x2 = __ldg(b2 + h);
    s0 += v.x * x0.x + v.y * x0.y;
    s1 += v.x * x1.x + v.y * x1.y;
    s2 += v.x * x2.x + v.y * x2.y;
  }
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if (lane == 0) {
    red[wid][0] = s0;
    red[wid][1] = s1;
    red[wid][2] = s2;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0.0;
    for (int w = 0; w < kDenseThreads / 32; ++w) t += red[w][threadIdx.x];
    F[row + threadIdx.x * n] = X::add(F[row + threadIdx.x * n], t);
  }
}

__global__ void __launch_bounds__(kDenseThreads) k_ivc_dense(IBArgs a, const double *rhs,
                                                             const double *Ainv, int ld, double *F) {
  dense_row(a, rhs, Ainv, ld, F, blockIdx.x);
}

// The same solve with A^-1 held in FP32 (the storage forms that keep their
// populations in 4 or 2 bytes): half the bytes per step, products and sums
// still in FP64; the rounding of A^-1 (2^-24 relative) is far below the
// populations' own.
__device__ __forceinline__ void dense_row32(const IBArgs &a, const double *rhs, const float *Ainv,
                                            int ld, double *F, int row) {
  __shared__ double red[kDenseThreads / 32][3];
  const int n = a.n;
  const int quarter = ld >> 2;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const float4 *Ar = reinterpret_cast<const float4 *>(Ainv + (size_t)row * ld);
  const double2 *b0 = reinterpret_cast<const double2 *>(rhs);
  const double2 *b1 = reinterpret_cast<const double2 *>(rhs + ld);
  const double2 *b2 = reinterpret_cast<const double2 *>(rhs + 2 * ld);
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll 4
  for (int h = threadIdx.x; h < quarter; h += kDenseThreads) {
    const float4 v = __ldcs(Ar + h);
    const double2 x0 = __ldg(b0 + 2 * h), y0 = __ldg(b0 + 2 * h + 1);
    const double2 x1 = __ldg(b1 + 2 * h), y1 = __ldg(b1 + 2 * h + 1);
    const double2 x2 = __ldg(b2 + 2 * h), y2 = __ldg(b2 + 2 * h + 1);
    s0 += double(v.x) * x0.x + double(v.y) * x0.y + double(v.z) * y0.x + double(v.w) * y0.y;
    s1 += double(v.x) * x1.x + double(v.y) * x1.y + double(v.z) * y1.x + double(v.w) * y1.y;
    s2 += double(v.x) * x2.x + double(v.y) * x2.y + double(v.z) * y2.x + double(v.w) * y2.y;
  }
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if (lane == 0) {
    red[wid][0] = s0;
    red[wid][1] = s1;
    red[wid][2] = s2;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0.0;
    for (int w = 0; w < kDenseThreads / 32; ++w) t += red[w][threadIdx.x];
    F[row + threadIdx.x * n] = X::add(F[row + threadIdx.x * n], t);
  }
}

__global__ void __launch_bounds__(kDenseThreads) k_ivc_dense32(IBArgs a, const double *rhs,
                                                               const float *Ainv, int ld, double *F) {
  dense_row32(a, rhs, Ainv, ld, F, blockIdx.x);
}

// kDenseRows rows per block: every thread has the loads of all its rows in
// flight at once and reads the right-hand side once for them, so the solve
// takes a quarter of the waves of one row per block.  TA: double or float A^-1.
constexpr int kDenseRows = 4;
template <class TA>
__global__ void __launch_bounds__(kDenseThreads) k_ivc_dense_rows(IBArgs a, const double *rhs,
                                                                  const TA *Ainv, int ld, double *F) {
  constexpr int V = 16 / (int)sizeof(TA);  // elements per 16-byte load
  __shared__ double red[kDenseThreads / 32][kDenseRows * 3];
  const int n = a.n, r0 = blockIdx.x * kDenseRows;
  const int nr = min(kDenseRows, n - r0);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double acc[kDenseRows][3];
#pragma unroll
  for (int r = 0; r < kDenseRows; ++r) acc[r][0] = acc[r][1] = acc[r][2] = 0.0;
  const int nv = ld / V;
  for (int h = threadIdx.x; h < nv; h += kDenseThreads) {
    double av[kDenseRows][V];
#pragma unroll
    for (int r = 0; r < kDenseRows; ++r) {
      const int row = r0 + min(r, nr - 1);  // rows past the end repeat the last one (unused)
      if (V == 2) {
        const double2 v = __ldcs(reinterpret_cast<const double2 *>(Ainv + (size_t)row * ld) + h);
        av[r][0] = v.x;
        av[r][1] = v.y;
      } else {
        const float4 v = __ldcs(reinterpret_cast<const float4 *>(Ainv + (size_t)row * ld) + h);
        av[r][0] = v.x;
        av[r][1] = v.y;
        av[r][V > 2 ? 2 : 0] = v.z;
        av[r][V > 3 ? 3 : 0] = v.w;
      }
    }
#pragma unroll
    for (int e = 0; e < V; ++e) {
      const int col = h * V + e;
      const double x0 = __ldg(rhs + col), x1 = __ldg(rhs + ld + col), x2 = __ldg(rhs + 2 * ld + col);
#pragma unroll
      for (int r = 0; r < kDenseRows; ++r) {
        acc[r][0] += av[r][e] * x0;
        acc[r][1] += av[r][e] * x1;
        acc[r][2] += av[r][e] * x2;
      }
    }
  }
#pragma unroll
  for (int r = 0; r < kDenseRows; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double x = acc[r][c];
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if (lane == 0) red[wid][r * 3 + c] = x;
    }
  __syncthreads();
  if ((int)threadIdx.x < nr * 3) {
    const int r = threadIdx.x / 3, c = threadIdx.x % 3;
    double t = 0.0;
    for (int w = 0; w < kDenseThreads / 32; ++w) t += red[w][threadIdx.x];
    F[r0 + r + c * n] = X::add(F[r0 + r + c * n], t);
  }
}

__global__ void __launch_bounds__(256) k_to_f32(const double *src, float *dst, int64_t n) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x)
    dst[t] = float(src[t]);
}

// force_spreading_cic, :1331-1448 (dv folded in, 2D spreads x and y only);
// one warp per marker, lanes over the stencil points, FP64 atomics; the
// marker's cell and lane's kernel weights (marker_weights) are given
__device__ __forceinline__ void spread_core(const IBArgs &a, int m, int lane, const double *F,
                                            double *EFI, int *status, int i0, int j0, int k0,
                                            double wxl, double wyl, double wzl) {
  const double fx = X::mul(F[m], a.dv), fy = X::mul(F[m + a.n], a.dv), fz = X::mul(F[m + 2 * a.n], a.dv);
  const double d = (a.dim == 3) ? X::mul(X::mul(a.dx[0], a.dx[1]), a.dx[2]) : X::mul(a.dx[0], a.dx[1]);
  const int ilo = a.dlo[0] - 2, ihi = a.dhi[0] + 2, jlo = a.dlo[1] - 2, jhi = a.dhi[1] + 2;
  const int klo = (a.dim == 3) ? a.dlo[2] - 2 : 0, khi = (a.dim == 3) ? a.dhi[2] + 2 : 0;
  const int npts = (a.dim == 3) ? 125 : 25;
  double scale = 1.0;
  if (a.renorm_spread) {
    double part = 0.0;
    for (int it = 0; it < (npts + 31) / 32; ++it) {
      const int t = lane + 32 * it;
      const int tt = t < npts ? t : 0;
      const int ii = tt / ((a.dim == 3) ? 25 : 5), jj = (tt / ((a.dim == 3) ? 5 : 1)) % 5;
      const int kk = (a.dim == 3) ? tt % 5 : 2;
      const double tU = __shfl_sync(0xffffffffu, wxl, ii, 32);
      const double tV = __shfl_sync(0xffffffffu, wyl, jj, 32);
      const double tW = __shfl_sync(0xffffffffu, wzl, kk, 32);
      if (t >= npts) continue;
      const int ip = i0 + ii - 2, jp = j0 + jj - 2, kp = (a.dim == 3) ? k0 + kk - 2 : 0;
      if (ip < ilo || ip > ihi || jp < jlo || jp > jhi || kp < klo || kp > khi) continue;
      const double t3 = (a.dim == 3) ? X::mul(X::mul(tU, tV), tW) : X::mul(tU, tV);
      part = X::add(part, X::mul(t3, d));
    }
    for (int o = 16; o > 0; o >>= 1) part = X::add(part, __shfl_xor_sync(0xffffffffu, part, o));
    if (part > 0.0) scale = X::div(1.0, part);
  }
  for (int it = 0; it < (npts + 31) / 32; ++it) {
    const int t = lane + 32 * it;
    const int tt = t < npts ? t : 0;
    const int ii = tt / ((a.dim == 3) ? 25 : 5), jj = (tt / ((a.dim == 3) ? 5 : 1)) % 5;
    const int kk = (a.dim == 3) ? tt % 5 : 2;
    const double tU = __shfl_sync(0xffffffffu, wxl, ii, 32);
    const double tV = __shfl_sync(0xffffffffu, wyl, jj, 32);
    const double tW = __shfl_sync(0xffffffffu, wzl, kk, 32);
    if (t >= npts) continue;
    const int ip = i0 + ii - 2, jp = j0 + jj - 2, kp = (a.dim == 3) ? k0 + kk - 2 : 0;
    if (ip < ilo || ip > ihi || jp < jlo || jp > jhi || kp < klo || kp > khi) continue;
    if (!in_band(a, ip, jp, kp)) {
      atomicOr(status, 1);
      continue;
    }
    const double t3 = (a.dim == 3) ? X::mul(X::mul(tU, tV), tW) : X::mul(tU, tV);
    // points outside the kernel's support would add signed zeros to a band
    // that starts at +0: skipping their atomics changes no value
    if (t3 == 0.0) continue;
    const double dvl = X::mul(t3, scale);
    const int64_t e = bidx(a, ip, jp, kp);
    atomicAdd(&EFI[e], X::mul(dvl, fx));
    atomicAdd(&EFI[e + a.nb], X::mul(dvl, fy));
    if (a.dim == 3) atomicAdd(&EFI[e + 2 * a.nb], X::mul(dvl, fz));
  }
}

__device__ __forceinline__ void spread_one(const IBArgs &a, int m, int lane, const double *xyz,
                                           const double *F, double *EFI, int *status) {
  int i0, j0, k0;
  double wxl, wyl, wzl;
  marker_weights(a, xyz[m], xyz[m + a.n], xyz[m + 2 * a.n], lane, i0, j0, k0, wxl, wyl, wzl);
  spread_core(a, m, lane, F, EFI, status, i0, j0, k0, wxl, wyl, wzl);
}

// the same from the step's weight table (kTabStride)
__device__ __forceinline__ void spread_one_tab(const IBArgs &a, int m, int lane, const double *tw,
                                               const int4 *tc, const double *F, double *EFI,
                                               int *status) {
  const double *row = tw + (int64_t)kTabStride * m;
  const int o = lane % 5;
  const int4 c = tc[m];
  spread_core(a, m, lane, F, EFI, status, c.x, c.y, c.z, row[o], row[5 + o], row[10 + o]);
}

// tw / tc: the step's weight table when the interpolation wrote one, else null
__global__ void __launch_bounds__(128) k_spread(IBArgs a, const double *xyz, const double *F,
                                                double *EFI, int *status, const double *tw,
                                                const int4 *tc) {
  const int lane = threadIdx.x & 31;
  const int m = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (m >= a.n) return;
  if (tc)
    spread_one_tab(a, m, lane, tw, tc, F, EFI, status);
  else
    spread_one(a, m, lane, xyz, F, EFI, status);
}

__global__ void __launch_bounds__(128) k_interp(IBArgs a, const double *xyz, const double *EV,
                                                double *uvw, int *status, const double *tgt,
                                                double *rhs, int ld, double *tw, int4 *tc) {
  const int lane = threadIdx.x & 31;
  const int m = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (m >= a.n) return;
  interp_one(a, m, lane, xyz, EV, uvw, status, tgt, rhs, ld, tw, tc);
}

// ---------------------------------------------------------------------------
// Interpolation and spreading in the reference's summation order.
// velocity_interpolation_cic sums a marker's stencil sequentially (i, then
// j, then k innermost, IBMarkerDF.cpp:612-695); force_spreading adds the
// markers' contributions to each cell in marker order (the loop over
// particles, :1331-1448).  The kernels below keep both orders: one thread per
// marker for the interpolation, and for a body whose markers do not move a
// gather over a cell -> marker table built once (markers in increasing
// order), so each cell's force is the reference's sum, computed once, with
// no atomics.  FP64 results then equal the reference's bit for bit wherever
// the rest of the chain does (explicit and explicit_diag coupling).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void interp_seq(const IBArgs &a, int m, const double *xyz,
                                           const double *EV, double *uvw, int *status,
                                           const double *tgt, double *rhs, int ld) {
  const double px = xyz[m], py = xyz[m + a.n], pz = xyz[m + 2 * a.n];
  const double d = (a.dim == 3) ? X::mul(X::mul(a.dx[0], a.dx[1]), a.dx[2]) : X::mul(a.dx[0], a.dx[1]);
  const int i0 = cell_of(px, a.plo[0], a.dx[0]), j0 = cell_of(py, a.plo[1], a.dx[1]);
  const int k0 = (a.dim == 3) ? cell_of(pz, a.plo[2], a.dx[2]) : 0;
  double wx[5], wy[5], wz[5];
#pragma unroll
  for (int o = 0; o < 5; ++o) {
    wx[o] = delta_fn(cell_center(a.plo[0], i0 + o - 2, a.dx[0]), px, a.dx[0], a.kt);
    wy[o] = delta_fn(cell_center(a.plo[1], j0 + o - 2, a.dx[1]), py, a.dx[1], a.kt);
    wz[o] = (a.dim == 3) ? delta_fn(cell_center(a.plo[2], k0 + o - 2, a.dx[2]), pz, a.dx[2], a.kt) : 1.0;
  }
  const int ilo = a.dlo[0] - 2, ihi = a.dhi[0] + 2, jlo = a.dlo[1] - 2, jhi = a.dhi[1] + 2;
  const int klo = (a.dim == 3) ? a.dlo[2] - 2 : 0, khi = (a.dim == 3) ? a.dhi[2] + 2 : 0;
  const int nk = (a.dim == 3) ? 5 : 1;
  double u = 0.0, v = 0.0, w = 0.0, part = 0.0;
  bool outside = false;
  for (int ii = 0; ii < 5; ++ii) {
    const int ip = i0 + ii - 2;
    if (ip < ilo || ip > ihi || wx[ii] == 0.0) continue;
    for (int jj = 0; jj < 5; ++jj) {
      const int jp = j0 + jj - 2;
      if (jp < jlo || jp > jhi || wy[jj] == 0.0) continue;
      for (int kk = 0; kk < nk; ++kk) {
        const int kp = (a.dim == 3) ? k0 + kk - 2 : 0;
        if (kp < klo || kp > khi) continue;
        const double dvl = (a.dim == 3) ? X::mul(X::mul(wx[ii], wy[jj]), wz[kk]) : X::mul(wx[ii], wy[jj]);
        // points outside the kernel's support add signed zeros to sums that
        // start at +0: skipping them leaves every sum bit for bit as it was
        if (dvl == 0.0) continue;
        if (!in_band(a, ip, jp, kp)) {
          outside = true;
          continue;
        }
        const int64_t e = bidx(a, ip, jp, kp);
        part = X::add(part, X::mul(dvl, d));
        u = X::add(u, X::mul(X::mul(dvl, EV[e]), d));
        v = X::add(v, X::mul(X::mul(dvl, EV[e + a.nb]), d));
        if (a.dim == 3) w = X::add(w, X::mul(X::mul(dvl, EV[e + 2 * a.nb]), d));
      }
    }
  }
  if (outside) atomicOr(status, 1);
  if (a.renorm_interp && part > 0.0) {
    u = X::div(u, part);
    v = X::div(v, part);
    w = X::div(w, part);
  }
  u = X::add(uvw[m], u);
  v = X::add(uvw[m + a.n], v);
  w = X::add(uvw[m + 2 * a.n], w);
  uvw[m] = u;
  uvw[m + a.n] = v;
  uvw[m + 2 * a.n] = w;
  if (rhs) {
    double Ux, Uy, Uz;
    target_of(a, m, xyz, tgt, Ux, Uy, Uz);
    rhs[m] = X::div(X::sub(Ux, u), a.dt);
    rhs[m + ld] = X::div(X::sub(Uy, v), a.dt);
    rhs[m + 2 * ld] = X::div(X::sub(Uz, w), a.dt);
  }
}

__global__ void __launch_bounds__(128) k_interp_seq(IBArgs a, const double *xyz, const double *EV,
                                                    double *uvw, int *status, const double *tgt,
                                                    double *rhs, int ld) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.n) return;
  interp_seq(a, m, xyz, EV, uvw, status, tgt, rhs, ld);
}

// per marker: its five kernel weights per direction and the spreading scale
// (1, or 1 / partition with renormalize_delta, the partition summed in the
// reference's order over the clipped stencil, :1336-1410)
struct SpreadW {
  double w[3][5];
  double scale;
};

__global__ void __launch_bounds__(128) k_spread_weights(IBArgs a, const double *xyz, SpreadW *W) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.n) return;
  const double p[3] = {xyz[m], xyz[m + a.n], xyz[m + 2 * a.n]};
  SpreadW sw;
  int c0[3];
  for (int dd = 0; dd < 3; ++dd) {
    c0[dd] = (dd < a.dim) ? cell_of(p[dd], a.plo[dd], a.dx[dd]) : 0;
    for (int o = 0; o < 5; ++o)
      sw.w[dd][o] = (dd < a.dim) ? delta_fn(cell_center(a.plo[dd], c0[dd] + o - 2, a.dx[dd]), p[dd],
                                             a.dx[dd], a.kt)
                                 : 1.0;
  }
  sw.scale = 1.0;
  if (a.renorm_spread) {
    const double d = (a.dim == 3) ? X::mul(X::mul(a.dx[0], a.dx[1]), a.dx[2]) : X::mul(a.dx[0], a.dx[1]);
    const int nk = (a.dim == 3) ? 5 : 1;
    double part = 0.0;
    for (int ii = 0; ii < 5; ++ii) {
      const int ip = c0[0] + ii - 2;
      if (ip < a.dlo[0] - 2 || ip > a.dhi[0] + 2) continue;
      for (int jj = 0; jj < 5; ++jj) {
        const int jp = c0[1] + jj - 2;
        if (jp < a.dlo[1] - 2 || jp > a.dhi[1] + 2) continue;
        for (int kk = 0; kk < nk; ++kk) {
          const int kp = c0[2] + kk - 2;
          if (a.dim == 3 && (kp < a.dlo[2] - 2 || kp > a.dhi[2] + 2)) continue;
          const double t3 = (a.dim == 3) ? X::mul(X::mul(sw.w[0][ii], sw.w[1][jj]), sw.w[2][kk])
                                         : X::mul(sw.w[0][ii], sw.w[1][jj]);
          part = X::add(part, X::mul(t3, d));
        }
      }
    }
    if (part > 0.0) sw.scale = X::div(1.0, part);
  }
  W[m] = sw;
}

// one thread per band cell that some stencil reaches: its markers' force
// contributions in increasing marker order.  ent: marker << 9 | ii << 6 |
// jj << 3 | kk.
// the force of gather row r: its markers' contributions in increasing order
__device__ __forceinline__ void gather_row(const IBArgs &a, const SpreadW *__restrict__ W,
                                           const double *__restrict__ F,
                                           const int *__restrict__ rowptr,
                                           const int *__restrict__ ent, int r, double &ax,
                                           double &ay, double &az) {
  ax = ay = az = 0.0;
  for (int e = rowptr[r]; e < rowptr[r + 1]; ++e) {
    const int pk = ent[e];
    const int m = pk >> 9, ii = (pk >> 6) & 7, jj = (pk >> 3) & 7, kk = pk & 7;
    const SpreadW &w = W[m];
    const double t3 = (a.dim == 3) ? X::mul(X::mul(w.w[0][ii], w.w[1][jj]), w.w[2][kk])
                                   : X::mul(w.w[0][ii], w.w[1][jj]);
    const double dvl = X::mul(t3, w.scale);
    ax = X::add(ax, X::mul(dvl, X::mul(F[m], a.dv)));
    ay = X::add(ay, X::mul(dvl, X::mul(F[m + a.n], a.dv)));
    if (a.dim == 3) az = X::add(az, X::mul(dvl, X::mul(F[m + 2 * a.n], a.dv)));
  }
}

__global__ void __launch_bounds__(128) k_spread_gather(IBArgs a, const SpreadW *__restrict__ W,
                                                       const double *__restrict__ F,
                                                       const int64_t *__restrict__ cells,
                                                       const int *__restrict__ rowptr,
                                                       const int *__restrict__ ent, int ncell,
                                                       double *EFI) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= ncell) return;
  double ax, ay, az;
  gather_row(a, W, F, rowptr, ent, r, ax, ay, az);
  const int64_t t = cells[r];
  EFI[t] = ax;
  EFI[t + a.nb] = ay;
  if (a.dim == 3) EFI[t + 2 * a.nb] = az;
}

// ---------------------------------------------------------------------------
// Interpolation and spreading of a body whose markers do not move, for the
// 4- and 2-byte storage forms: the markers' kernel weights come from the
// table computed once (k_spread_weights), lane l < 15 of the marker's warp
// holding weight l % 5 of direction l / 5 and lane 15 the spreading scale, so
// no kernel value is evaluated per step; the sums are left to fused
// multiply-adds, whose rounding lies far below those forms' own precision.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double table_weight(const SpreadW *W, int m, int lane) {
  return (lane < 16) ? reinterpret_cast<const double *>(W + m)[lane] : 0.0;
}

// fresh: the markers' velocities and forces start from zero here (the
// zeroing of k_markers, for bodies whose positions need no update)
__global__ void __launch_bounds__(128) k_interp_w(IBArgs a, const double *xyz,
                                                  const SpreadW *__restrict__ W,
                                                  const double *__restrict__ EV, double *uvw,
                                                  double *F, int fresh, int *status,
                                                  const double *tgt, double *rhs, int ld) {
  const int lane = threadIdx.x & 31;
  const int m = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (m >= a.n) return;
  const double wl = table_weight(W, m, lane);
  const int i0 = cell_of(xyz[m], a.plo[0], a.dx[0]), j0 = cell_of(xyz[m + a.n], a.plo[1], a.dx[1]);
  const int k0 = (a.dim == 3) ? cell_of(xyz[m + 2 * a.n], a.plo[2], a.dx[2]) : 0;
  const double d = (a.dim == 3) ? a.dx[0] * a.dx[1] * a.dx[2] : a.dx[0] * a.dx[1];
  const int ilo = a.dlo[0] - 2, ihi = a.dhi[0] + 2, jlo = a.dlo[1] - 2, jhi = a.dhi[1] + 2;
  const int klo = (a.dim == 3) ? a.dlo[2] - 2 : 0, khi = (a.dim == 3) ? a.dhi[2] + 2 : 0;
  const int npts = (a.dim == 3) ? 125 : 25;
  double u = 0.0, v = 0.0, w = 0.0, part = 0.0;
  const int nit = (npts + 31) / 32;
  for (int it = 0; it < nit; ++it) {
    const int t = lane + 32 * it;
    const int tt = t < npts ? t : 0;
    const int ii = tt / ((a.dim == 3) ? 25 : 5), jj = (tt / ((a.dim == 3) ? 5 : 1)) % 5;
    const int kk = (a.dim == 3) ? tt % 5 : 2;
    const double tU = __shfl_sync(0xffffffffu, wl, ii, 32);
    const double tV = __shfl_sync(0xffffffffu, wl, 5 + jj, 32);
    const double tW = __shfl_sync(0xffffffffu, wl, 10 + kk, 32);
    if (t >= npts) continue;
    const int ip = i0 + ii - 2, jp = j0 + jj - 2, kp = (a.dim == 3) ? k0 + kk - 2 : 0;
    if (ip < ilo || ip > ihi || jp < jlo || jp > jhi || kp < klo || kp > khi) continue;
    if (!in_band(a, ip, jp, kp)) {
      atomicOr(status, 1);
      continue;
    }
    const double dvl = tU * tV * tW;
    if (dvl == 0.0) continue;
    const int64_t e = bidx(a, ip, jp, kp);
    const double dd = dvl * d;
    part += dd;
    u = fma(dd, EV[e], u);
    v = fma(dd, EV[e + a.nb], v);
    if (a.dim == 3) w = fma(dd, EV[e + 2 * a.nb], w);
  }
  for (int o = 16; o > 0; o >>= 1) {
    u += __shfl_down_sync(0xffffffffu, u, o);
    v += __shfl_down_sync(0xffffffffu, v, o);
    w += __shfl_down_sync(0xffffffffu, w, o);
    part += __shfl_down_sync(0xffffffffu, part, o);
  }
  if (lane == 0) {
    if (a.renorm_interp && part > 0.0) {
      u /= part;
      v /= part;
      w /= part;
    }
    if (fresh) {
      F[m] = 0.0;
      F[m + a.n] = 0.0;
      F[m + 2 * a.n] = 0.0;
    } else {
      u += uvw[m];
      v += uvw[m + a.n];
      w += uvw[m + 2 * a.n];
    }
    uvw[m] = u;
    uvw[m + a.n] = v;
    uvw[m + 2 * a.n] = w;
    if (rhs) {
      double Ux, Uy, Uz;
      target_of(a, m, xyz, tgt, Ux, Uy, Uz);
      rhs[m] = (Ux - u) / a.dt;
      rhs[m + ld] = (Uy - v) / a.dt;
      rhs[m + 2 * ld] = (Uz - w) / a.dt;
    }
  }
}

__global__ void __launch_bounds__(128) k_spread_w(IBArgs a, const double *xyz,
                                                  const SpreadW *__restrict__ W, const double *F,
                                                  double *EFI, int *status) {
  const int lane = threadIdx.x & 31;
  const int m = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (m >= a.n) return;
  const double wl = table_weight(W, m, lane);
  const double scale = __shfl_sync(0xffffffffu, wl, 15, 32);
  const int i0 = cell_of(xyz[m], a.plo[0], a.dx[0]), j0 = cell_of(xyz[m + a.n], a.plo[1], a.dx[1]);
  const int k0 = (a.dim == 3) ? cell_of(xyz[m + 2 * a.n], a.plo[2], a.dx[2]) : 0;
  const double fx = F[m] * a.dv * scale, fy = F[m + a.n] * a.dv * scale;
  const double fz = F[m + 2 * a.n] * a.dv * scale;
  const int ilo = a.dlo[0] - 2, ihi = a.dhi[0] + 2, jlo = a.dlo[1] - 2, jhi = a.dhi[1] + 2;
  const int klo = (a.dim == 3) ? a.dlo[2] - 2 : 0, khi = (a.dim == 3) ? a.dhi[2] + 2 : 0;
  const int npts = (a.dim == 3) ? 125 : 25;
  const int nit = (npts + 31) / 32;
  for (int it = 0; it < nit; ++it) {
    const int t = lane + 32 * it;
    const int tt = t < npts ? t : 0;
    const int ii = tt / ((a.dim == 3) ? 25 : 5), jj = (tt / ((a.dim == 3) ? 5 : 1)) % 5;
    const int kk = (a.dim == 3) ? tt % 5 : 2;
    const double tU = __shfl_sync(0xffffffffu, wl, ii, 32);
    const double tV = __shfl_sync(0xffffffffu, wl, 5 + jj, 32);
    const double tW = __shfl_sync(0xffffffffu, wl, 10 + kk, 32);
    if (t >= npts) continue;
    const int ip = i0 + ii - 2, jp = j0 + jj - 2, kp = (a.dim == 3) ? k0 + kk - 2 : 0;
    if (ip < ilo || ip > ihi || jp < jlo || jp > jhi || kp < klo || kp > khi) continue;
    if (!in_band(a, ip, jp, kp)) {
      atomicOr(status, 1);
      continue;
    }
    const double t3 = tU * tV * tW;
    if (t3 == 0.0) continue;
    const int64_t e = bidx(a, ip, jp, kp);
    atomicAdd(&EFI[e], t3 * fx);
    atomicAdd(&EFI[e + a.nb], t3 * fy);
    if (a.dim == 3) atomicAdd(&EFI[e + 2 * a.nb], t3 * fz);
  }
}

// SumBoundary (periodic): ghost-cell contributions added into their valid image
__device__ __forceinline__ void sum_boundary_cell(const IBArgs &a, double *EFI, int64_t t) {
  {
    const int i = a.blo[0] + (int)(t % a.bn[0]);
    const int j = a.blo[1] + (int)((t / a.bn[0]) % a.bn[1]);
    const int k = a.blo[2] + (int)(t / ((int64_t)a.bn[0] * a.bn[1]));
    const int g[3] = {i, j, k};
    bool inside = true;
    for (int d = 0; d < a.dim; ++d) inside = inside && g[d] >= a.dlo[d] && g[d] <= a.dhi[d];
    if (!inside) return;
    // visit every periodic image of this cell that lies in the band
    int nsh[3] = {1, 1, 1};
    for (int d = 0; d < a.dim; ++d) nsh[d] = a.periodic[d] ? 3 : 1;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int sx = 0; sx < nsh[0]; ++sx)
      for (int sy = 0; sy < nsh[1]; ++sy)
        for (int sz = 0; sz < nsh[2]; ++sz) {
          if (sx == 0 && sy == 0 && sz == 0) continue;
          const int off[3] = {sx == 1 ? 1 : (sx == 2 ? -1 : 0), sy == 1 ? 1 : (sy == 2 ? -1 : 0),
                              sz == 1 ? 1 : (sz == 2 ? -1 : 0)};
          int h[3] = {i, j, k};
          for (int d = 0; d < a.dim; ++d) h[d] += off[d] * (a.dhi[d] - a.dlo[d] + 1);
          if (!in_band(a, h[0], h[1], h[2])) continue;
          const int64_t e = bidx(a, h[0], h[1], h[2]);
          for (int c = 0; c < 3; ++c) acc[c] = X::add(acc[c], EFI[e + c * a.nb]);
        }
    for (int c = 0; c < 3; ++c) EFI[t + c * a.nb] = X::add(EFI[t + c * a.nb], acc[c]);
  }
}

__global__ void k_sum_boundary(IBArgs a, double *EFI) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < a.nb;
       t += (int64_t)gridDim.x * blockDim.x)
    sum_boundary_cell(a, EFI, t);
}

// marker force sum (:1781-1819), deterministic single-CTA reduction
// Fixed-order sum of the marker forces times dv: each thread takes markers
// t, t + B, t + 2B, ... in two interleaved chains (even and odd multiples of
// B), the three components together, then one block reduction per component.
__device__ __forceinline__ void marker_sum_block(const IBArgs &a, const double *F, double *fsum) {
  __shared__ double sh[33];
  double s0[3] = {0.0, 0.0, 0.0}, s1[3] = {0.0, 0.0, 0.0};
  const int B = blockDim.x;
  int m = threadIdx.x;
  for (; m + B < a.n; m += 2 * B) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      s0[c] = X::add(s0[c], X::mul(F[m + c * a.n], a.dv));
      s1[c] = X::add(s1[c], X::mul(F[m + B + c * a.n], a.dv));
    }
  }
  if (m < a.n) {
#pragma unroll
    for (int c = 0; c < 3; ++c) s0[c] = X::add(s0[c], X::mul(F[m + c * a.n], a.dv));
  }
  for (int c = 0; c < 3; ++c) {
    const double t = block_sum(X::add(s0[c], s1[c]), sh);
    if (threadIdx.x == 0) fsum[c] = X::add(fsum[c], t);
  }
}

__global__ void __launch_bounds__(1024) k_marker_sum(IBArgs a, const double *F, double *fsum) {
  marker_sum_block(a, F, fsum);
}

// velocity_correction (valid cells) and EulerForceTotal += EulerForceIter, :1878-1879;
// then FillBoundary of the periodic band ghosts of EV
__global__ void k_correct(IBArgs a, double *EV, const double *EFI, double *EFT) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < a.nb;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int i = a.blo[0] + (int)(t % a.bn[0]);
    const int j = a.blo[1] + (int)((t / a.bn[0]) % a.bn[1]);
    const int k = a.blo[2] + (int)(t / ((int64_t)a.bn[0] * a.bn[1]));
    const int g[3] = {i, j, k};
    bool inside = true;
    for (int d = 0; d < a.dim; ++d) inside = inside && g[d] >= a.dlo[d] && g[d] <= a.dhi[d];
    if (!inside) continue;
    for (int c = 0; c < 3; ++c) {
      EV[t + c * a.nb] = X::add(EV[t + c * a.nb], X::mul(a.dt, EFI[t + c * a.nb]));
      EFT[t + c * a.nb] = X::add(EFT[t + c * a.nb], EFI[t + c * a.nb]);
    }
  }
}

__device__ __forceinline__ void fill_boundary_cell(const IBArgs &a, double *EV, int64_t t) {
  {
    int g[3];
    g[0] = a.blo[0] + (int)(t % a.bn[0]);
    g[1] = a.blo[1] + (int)((t / a.bn[0]) % a.bn[1]);
    g[2] = a.blo[2] + (int)(t / ((int64_t)a.bn[0] * a.bn[1]));
    bool inside = true, wrappable = true;
    for (int d = 0; d < a.dim; ++d) {
      const bool out = g[d] < a.dlo[d] || g[d] > a.dhi[d];
      if (out) {
        inside = false;
        if (!a.periodic[d]) wrappable = false;
      }
    }
    if (inside || !wrappable) return;
    int w[3] = {g[0], g[1], g[2]};
    for (int d = 0; d < a.dim; ++d) {
      const int nn = a.dhi[d] - a.dlo[d] + 1;
      w[d] = a.dlo[d] + (((w[d] - a.dlo[d]) % nn) + nn) % nn;
    }
    if (!in_band(a, w[0], w[1], w[2])) return;
    const int64_t e = bidx(a, w[0], w[1], w[2]);
    for (int c = 0; c < 3; ++c) EV[t + c * a.nb] = EV[e + c * a.nb];
  }
}

__global__ void k_fill_boundary(IBArgs a, double *EV) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < a.nb;
       t += (int64_t)gridDim.x * blockDim.x)
    fill_boundary_cell(a, EV, t);
}

// export, :1889-1911: F = dt * rho * a on valid band cells
template <class R>
__device__ __forceinline__ void export_cell(const IBArgs &a, const double *EFT, const double *RHO,
                                            R *F, int mgl0, int mgl1, int mgl2, int64_t ms0,
                                            int64_t ms1, int64_t ms2, int64_t t,
                                            double *stored = nullptr) {
  const int i = a.blo[0] + (int)(t % a.bn[0]);
  const int j = a.blo[1] + (int)((t / a.bn[0]) % a.bn[1]);
  const int k = a.blo[2] + (int)(t / ((int64_t)a.bn[0] * a.bn[1]));
  const int g[3] = {i, j, k};
  bool inside = true;
  for (int d = 0; d < a.dim; ++d) inside = inside && g[d] >= a.dlo[d] && g[d] <= a.dhi[d];
  if (!inside) return;
  const int64_t m = (int64_t)(i - mgl0) + (int64_t)(j - mgl1) * ms0 + (int64_t)(k - mgl2) * ms1;
  const double dr = X::mul(a.dt, RHO[t]);
  const R fx = R(X::mul(dr, EFT[t])), fy = R(X::mul(dr, EFT[t + a.nb]));
  F[m] = fx;
  F[m + ms2] = fy;
  R fz = R(0);
  if (a.dim == 3) {
    fz = R(X::mul(dr, EFT[t + 2 * a.nb]));
    F[m + 2 * ms2] = fz;
  }
  if (stored) {  // the values as stored (the force region is the band inside the domain)
    stored[0] = double(fx);
    stored[1] = double(fy);
    stored[2] = double(fz);
  }
}

template <class R>
__global__ void k_export(IBArgs a, const double *EFT, const double *RHO, R *F, int mgl0,
                         int mgl1, int mgl2, int64_t ms0, int64_t ms1, int64_t ms2) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < a.nb;
       t += (int64_t)gridDim.x * blockDim.x)
    export_cell<R>(a, EFT, RHO, F, mgl0, mgl1, mgl2, ms0, ms1, ms2, t);
}

// export to a level held in several boxes: the force of a band cell goes to
// the box whose valid region holds it (cells no box holds are dropped, as
// the reference's SumBoundary drops spread force outside the level's valid
// cells, IBMarkerDF.cpp:1511) and, as FillBoundary of the force before the
// collision does (Source/Core/AdvanceLBMAtLevel.cpp:187-194), to every box
// whose grown force array holds the cell or one of its periodic images as a
// ghost.
template <class R>
__global__ void k_export_boxes(IBArgs a, const double *EFT, const double *RHO,
                               const StepArgs *__restrict__ args, int nargs) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < a.nb;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int g[3] = {a.blo[0] + (int)(t % a.bn[0]), a.blo[1] + (int)((t / a.bn[0]) % a.bn[1]),
                      a.blo[2] + (int)(t / ((int64_t)a.bn[0] * a.bn[1]))};
    bool inside = true;
    for (int d = 0; d < a.dim; ++d) inside = inside && g[d] >= a.dlo[d] && g[d] <= a.dhi[d];
    if (!inside) continue;
    bool owned = false;
    for (int b = 0; b < nargs && !owned; ++b) {
      const StepArgs &x = args[b];
      owned = g[0] >= x.lo[0] && g[0] <= x.hi[0] && g[1] >= x.lo[1] && g[1] <= x.hi[1] &&
              (a.dim == 2 || (g[2] >= x.lo[2] && g[2] <= x.hi[2]));
    }
    if (!owned) continue;
    const double dr = X::mul(a.dt, RHO[t]);
    const R fx = R(X::mul(dr, EFT[t])), fy = R(X::mul(dr, EFT[t + a.nb]));
    const R fz = R(a.dim == 3 ? X::mul(dr, EFT[t + 2 * a.nb]) : 0.0);
    // shifts by whole domain lengths along periodic directions (0 included)
    const int n[3] = {a.dhi[0] - a.dlo[0] + 1, a.dhi[1] - a.dlo[1] + 1, a.dhi[2] - a.dlo[2] + 1};
    for (int s = 0; s < 27; ++s) {
      const int sh[3] = {s % 3 - 1, (s / 3) % 3 - 1, s / 9 - 1};
      bool ok = true;
      for (int d = 0; d < 3; ++d)
        if (sh[d] != 0 && (d >= a.dim || !a.periodic[d])) ok = false;
      if (!ok) continue;
      const int c[3] = {g[0] + sh[0] * n[0], g[1] + sh[1] * n[1], g[2] + sh[2] * n[2]};
      for (int b = 0; b < nargs; ++b) {
        const StepArgs &x = args[b];
        bool in = true;
        for (int d = 0; d < a.dim; ++d) {
          const int w = x.lo[d] - x.mgl[d];
          in = in && c[d] >= x.lo[d] - w && c[d] <= x.hi[d] + w;
        }
        if (!in) continue;
        R *F = static_cast<R *>(const_cast<void *>(x.force));
        const int64_t m = (int64_t)(c[0] - x.mgl[0]) + (int64_t)(c[1] - x.mgl[1]) * x.ms0 +
                          (int64_t)(a.dim == 3 ? c[2] - x.mgl[2] : 0) * x.ms1;
        F[m] = fx;
        F[m + x.ms2] = fy;
        if (a.dim == 3) F[m + 2 * x.ms2] = fz;
      }
    }
  }
}


}  // namespace

// ---------------------------------------------------------------------------
// Host object
// ---------------------------------------------------------------------------
struct ilbm_ib {
  ilbm_ctx *ctx = nullptr;
  ilbm_ib_params p{};
  ilbm_level_geom g{};
  int dim = 2, kt = 0, n = 0;
  double dv = 0, wall_tol = 0;
  double dx[3] = {0, 0, 0};
  bool moving = false;
  std::vector<double> xref, yref, zref;  // 1-based (index 0 unused)
  std::vector<double> hx, hy, hz;        // static positions
  int blo[3] = {0, 0, 0}, bn[3] = {1, 1, 1};
  int64_t nb = 0;
  double *d_xyz = nullptr, *d_ref = nullptr, *d_tgt = nullptr, *d_uvw = nullptr, *d_F = nullptr;
  double *d_EV = nullptr, *d_EFI = nullptr, *d_EFT = nullptr, *d_RHO = nullptr;
  double *d_fsum = nullptr;
  int *d_status = nullptr, *d_iters = nullptr;
  int *d_rowptr = nullptr, *d_col = nullptr;
  double *d_val = nullptr, *d_diag = nullptr, *d_X = nullptr, *d_work = nullptr;
  int nnz_cap = 0;
  bool csr_ready = false;
  double *d_partial = nullptr;  // CG block partials
  int cg_blocks = 0;
  // the IVC solutions the next CG start may use (device int, 0-2): d_X the
  // last, d_Xh the one before it; the solves themselves advance it
  int *d_hist = nullptr;
  double *d_Xh = nullptr;
  // fixed operator solved through its stored inverse (k_ivc_dense)
  int ivc_solver = ILBM_IVC_AUTO;
  bool dense = false, dense_ready = false;
  int ld = 0;
  double *d_Ainv = nullptr, *d_gj = nullptr, *d_rhs = nullptr;
  float *d_Ainv32 = nullptr;  // FP32 copy of A^-1 for the 4- and 2-byte storage forms
  bool fsum_deferred = false;  // marker force sum still to be launched (ib_finish)
  // fixed-order spreading of a body whose markers do not move: the band cells
  // its stencils reach, their marker lists (CSR) and the markers' weights
  bool gather = false;
  int gather_cells = 0;
  int64_t *d_gcell = nullptr;
  int *d_growptr = nullptr, *d_gent = nullptr;
  void *d_sw = nullptr;  // SpreadW per marker
  bool sw_ready = false;  // d_sw holds the (fixed) markers' weights
  // a step's marker weight table (kTabStride per marker) and cells, written
  // by the warp-parallel interpolation for the spreading and operator build
  double *d_tw = nullptr;
  int4 *d_tc = nullptr;
  double *d_recscr = nullptr;  // scratch of a force record taken with the step
  // a level held in several boxes: the StepArgs of the boxes near the band
  std::vector<StepArgs> h_boxargs;
  StepArgs *d_boxargs = nullptr;
  int boxargs_cap = 0;
  std::vector<void *> allocs;
};

namespace {

template <class T>
int dmalloc(ilbm_ib *ib, T **p, size_t count) {
  void *q = nullptr;
  cudaError_t e = ilbm_ctx_malloc(ib->ctx, &q, count * sizeof(T));
  if (e != cudaSuccess) return cuda_fail(e, "device allocation (IB)");
  ib->allocs.push_back(q);
  *p = static_cast<T *>(q);
  return ILBM_OK;
}

int kernel_of(int t) {
  if (t == 4 || t == 0) return 0;
  if (t == 3 || t == 1) return 1;
  return 0;
}

// build_markers, IBMarkerDF.cpp:201-497 (+ IBMUserDefinedGeometry.H:59-142)
int build_markers(ilbm_ib *ib) {
  const ilbm_ib_params &p = ib->p;
  const ilbm_level_geom &g = ib->g;
  const double h = ib->dx[0];
  int Ml = p.n_marker;
  double dv = 0.0;
  std::vector<double> phi, theta;
  if (p.geometry_type == 1) {
    if (ib->dim != 2) {
      set_error("box marker geometry is implemented for 2D only");
      return ILBM_ERR_UNSUPPORTED;
    }
    double xlo = p.box_xlo, xhi = p.box_xhi, ylo = p.box_ylo, yhi = p.box_yhi;
    if (xhi <= xlo) { xlo = g.prob_lo[0]; xhi = g.prob_hi[0]; }
    if (yhi <= ylo) { ylo = g.prob_lo[1]; yhi = g.prob_hi[1]; }
    const double epsx = std::max(1.0e-6 * ib->dx[0], 1.0e-12);
    const double epsy = std::max(1.0e-6 * ib->dx[1], 1.0e-12);
    xlo = std::max(xlo, g.prob_lo[0] + epsx);
    xhi = std::min(xhi, g.prob_hi[0] - epsx);
    ylo = std::max(ylo, g.prob_lo[1] + epsy);
    yhi = std::min(yhi, g.prob_hi[1] - epsy);
    if (xhi <= xlo || yhi <= ylo) {
      set_error("invalid in-domain box bounds after clamping");
      return ILBM_ERR_ARG;
    }
    ib->p.box_xlo = xlo; ib->p.box_xhi = xhi; ib->p.box_ylo = ylo; ib->p.box_yhi = yhi;
    double ds = (p.box_ds > 0.0) ? p.box_ds : h;
    ds = std::max(ds, 1.0e-12);
    const int nx = std::max(2, (int)std::lround((xhi - xlo) / ds) + 1);
    const int ny = std::max(2, (int)std::lround((yhi - ylo) / ds) + 1);
    const double dsx = (xhi - xlo) / double(nx - 1), dsy = (yhi - ylo) / double(ny - 1);
    const bool lid = p.box_lid_only != 0;
    ib->xref.assign(1, 0.0); ib->yref.assign(1, 0.0); ib->zref.assign(1, 0.0);
    auto add = [&](double x, double y) { ib->xref.push_back(x); ib->yref.push_back(y); ib->zref.push_back(0.0); };
    if (lid) {
      for (int i = 0; i < nx; ++i) add(xlo + double(i) * dsx, yhi);
    } else {
      for (int i = 0; i < nx; ++i) add(xlo + double(i) * dsx, ylo);
      for (int i = 0; i < nx; ++i) add(xlo + double(i) * dsx, yhi);
      for (int j = 1; j < ny - 1; ++j) {
        const double y = ylo + double(j) * dsy;
        add(xlo, y);
        add(xhi, y);
      }
    }
    Ml = (int)ib->xref.size() - 1;
    const double per = lid ? (xhi - xlo) : 2.0 * ((xhi - xlo) + (yhi - ylo));
    dv = (per / double(Ml)) * h;
    ib->wall_tol = (p.box_wall_tol > 0.0) ? p.box_wall_tol : std::max(0.25 * std::min(dsx, dsy), 1.0e-12);
  } else if (p.geometry_type == 2) {
    if (ib->dim != 2) {
      set_error("user-defined (pitching NACA) geometry is implemented for 2D only");
      return ILBM_ERR_UNSUPPORTED;
    }
    const double chord = std::max(p.airfoil_chord, 1.0e-12);
    const double thick = std::max(p.airfoil_thickness, 1.0e-12);
    const int n_half = (p.n_marker > 0) ? std::max(p.n_marker / 2, 32)
                                        : std::max((int)std::ceil(1.5 * chord / h), 48);
    ib->xref.assign(1, 0.0); ib->yref.assign(1, 0.0); ib->zref.assign(1, 0.0);
    auto prof = [&](double x) {
      const double xc = std::min(std::max(x / chord, 0.0), 1.0);
      const double sx = std::sqrt(std::max(xc, 0.0));
      return 5.0 * thick * chord *
             (0.2969 * sx - 0.1260 * xc - 0.3516 * xc * xc + 0.2843 * xc * xc * xc -
              0.1036 * xc * xc * xc * xc);
    };
    for (int i = 0; i <= n_half; ++i) {
      const double beta = kPi * double(i) / double(n_half);
      const double x = 0.5 * chord * (1.0 - std::cos(beta));
      ib->xref.push_back(x); ib->yref.push_back(prof(x)); ib->zref.push_back(0.0);
    }
    for (int i = n_half - 1; i >= 1; --i) {
      const double beta = kPi * double(i) / double(n_half);
      const double x = 0.5 * chord * (1.0 - std::cos(beta));
      ib->xref.push_back(x); ib->yref.push_back(-prof(x)); ib->zref.push_back(0.0);
    }
    Ml = (int)ib->xref.size() - 1;
    double per = 0.0;
    for (int i = 1; i <= Ml; ++i) {
      const int in = (i == Ml) ? 1 : i + 1;
      const double a = ib->xref[in] - ib->xref[i], b = ib->yref[in] - ib->yref[i];
      per += std::sqrt(a * a + b * b);
    }
    dv = (per / double(Ml)) * h;
    ib->wall_tol = 0.0;
    ib->moving = true;
  } else if (ib->dim == 2) {
    if (Ml <= 0) {
      Ml = (int)std::ceil(2.0 * kPi * p.R / h);
      Ml = std::max(Ml, 16);
    }
    dv = (2.0 * kPi * p.R * h) / double(Ml);
    phi.assign(Ml + 1, 0.0);
    theta.assign(Ml + 1, 0.5 * kPi);
    for (int i = 1; i <= Ml; ++i) phi[i] = 2.0 * kPi * double(i - 1) / double(Ml);
  } else {
    const double t1 = p.R - (p.rd - 0.5) * h, t2 = p.R - (p.rd + 0.5) * h;
    const double a1 = t1 * (t1 * t1), a2 = t2 * (t2 * t2);
    if (Ml <= 0) {
      const double denom = 3.0 * h * h * h / 4.0 / kPi;
      Ml = (int)((a1 - a2) / denom);
      Ml = std::max(Ml, 32);
    }
    dv = (a1 - a2) / (3.0 * double(Ml) / 4.0 / kPi);
    phi.assign(Ml + 1, 0.0);
    theta.assign(Ml + 1, 0.0);
    double ph = 0.0;
    for (int mi = 0; mi < Ml; ++mi) {
      const double Hk = -1.0 + 2.0 * double(mi) / (double(Ml) - 1.0);
      const double th = std::acos(Hk);
      if (mi == 0 || mi == Ml - 1) ph = 0.0;
      else ph = std::fmod(ph + 3.809 / std::sqrt(double(Ml)) / std::sqrt(1.0 - Hk * Hk), 2.0 * kPi);
      phi[mi + 1] = ph;
      theta[mi + 1] = th;
    }
  }
  ib->n = Ml;
  ib->dv = dv;
  // static positions (update_lagrangian_marker / gather_marker_state formulas)
  ib->hx.assign(Ml, 0.0); ib->hy.assign(Ml, 0.0); ib->hz.assign(Ml, 0.0);
  for (int i = 0; i < Ml; ++i) {
    const int idx = i + 1;
    double x, y, z;
    if (p.geometry_type == 1) {
      x = ib->xref[idx]; y = ib->yref[idx]; z = 0.0;
    } else if (p.geometry_type == 2) {
      // placeholder; moving markers are positioned on the device each call
      x = p.x0 + ib->xref[idx] - p.pivot_x; y = p.y0 + ib->yref[idx]; z = 0.0;
    } else {
      x = p.x0 + p.R * std::sin(theta[idx]) * std::cos(phi[idx]);
      y = p.y0 + p.R * std::sin(theta[idx]) * std::sin(phi[idx]);
      z = (ib->dim == 3) ? p.z0 + p.R * std::cos(theta[idx]) : 0.0;
    }
    double pos[3] = {x, y, z};
    for (int d = 0; d < ib->dim; ++d) {
      if (!g.periodic[d]) continue;
      const double L = g.prob_hi[d] - g.prob_lo[d];
      while (pos[d] < g.prob_lo[d]) pos[d] += L;
      while (pos[d] >= g.prob_hi[d]) pos[d] -= L;
    }
    ib->hx[i] = pos[0]; ib->hy[i] = pos[1]; ib->hz[i] = pos[2];
  }
  return ILBM_OK;
}

// support band: marker envelope + 3 cells, clipped to the domain grown by 2;
// periodic directions the band touches are widened to the whole domain so
// every periodic image of a stencil cell is in the band.
void build_band(ilbm_ib *ib) {
  const ilbm_level_geom &g = ib->g;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  auto take = [&](double x, double y, double z) {
    const double v[3] = {x, y, z};
    for (int d = 0; d < 3; ++d) { lo[d] = std::min(lo[d], v[d]); hi[d] = std::max(hi[d], v[d]); }
  };
  if (ib->moving) {
    double rmax = 0.0;
    for (size_t i = 1; i < ib->xref.size(); ++i) {
      const double xr = ib->xref[i] - ib->p.pivot_x, yr = ib->yref[i];
      rmax = std::max(rmax, std::sqrt(xr * xr + yr * yr));
    }
    take(ib->p.x0 - rmax, ib->p.y0 - rmax, ib->p.z0);
    take(ib->p.x0 + rmax, ib->p.y0 + rmax, ib->p.z0);
  } else {
    for (int i = 0; i < ib->n; ++i) take(ib->hx[i], ib->hy[i], ib->hz[i]);
  }
  for (int d = 0; d < 3; ++d) {
    if (d >= ib->dim) { ib->blo[d] = 0; ib->bn[d] = 1; continue; }
    const int nd = g.n_cell[d];
    int a = (int)std::floor((lo[d] - g.prob_lo[d]) / ib->dx[d]) - 3;
    int b = (int)std::floor((hi[d] - g.prob_lo[d]) / ib->dx[d]) + 3;
    a = std::max(a, -2);
    b = std::min(b, nd - 1 + 2);
    if (g.periodic[d] && (a < 2 || b > nd - 3)) { a = -2; b = nd + 1; }
    ib->blo[d] = a;
    ib->bn[d] = b - a + 1;
  }
  ib->nb = (int64_t)ib->bn[0] * ib->bn[1] * ib->bn[2];
}

// The cell -> marker table of the fixed-order spreading (k_spread_gather)
// for a body whose markers do not move: every band cell within the kernel's
// support of a marker, with its markers in increasing order.  The host
// repeats the device's cell and distance arithmetic (IEEE double, no
// contraction), so the table holds exactly the stencil points whose weight
// is nonzero (plus, at worst, a few of weight zero, which add signed zeros).
int build_gather(ilbm_ib *ib) {
  const int n = ib->n, dim = ib->dim;
  if (ib->moving || n <= 0 || n >= (1 << 22)) return ILBM_OK;
  const double R = (ib->kt == 0) ? 2.0 : 1.5;
  const ilbm_level_geom &g = ib->g;
  std::vector<std::pair<int64_t, int>> pairs;
  pairs.reserve((size_t)n * (dim == 3 ? 64 : 16));
  for (int m = 0; m < n; ++m) {
    const double p[3] = {ib->hx[m], ib->hy[m], ib->hz[m]};
    int c0[3] = {0, 0, 0};
    bool sup[3][5];
    for (int d = 0; d < 3; ++d)
      for (int o = 0; o < 5; ++o) sup[d][o] = (d >= dim && o == 2);
    for (int d = 0; d < dim; ++d) {
      c0[d] = (int)std::floor((p[d] - g.prob_lo[d]) / ib->dx[d]);
      for (int o = 0; o < 5; ++o) {
        const double xc = g.prob_lo[d] + ((double)(c0[d] + o - 2) + 0.5) * ib->dx[d];
        const double rr = std::fabs(xc - p[d]) / ib->dx[d];
        sup[d][o] = rr < R * (1.0 + 1e-12);
      }
    }
    for (int ii = 0; ii < 5; ++ii)
      for (int jj = 0; jj < 5; ++jj)
        for (int kk = 0; kk < 5; ++kk) {
          if (!sup[0][ii] || !sup[1][jj] || !sup[2][kk]) continue;
          const int c[3] = {c0[0] + ii - 2, c0[1] + jj - 2, dim == 3 ? c0[2] + kk - 2 : 0};
          bool ok = true;
          for (int d = 0; d < dim; ++d) {
            if (c[d] < -2 || c[d] > g.n_cell[d] + 1) ok = false;  // clip: domain grown by 2
            if (c[d] < ib->blo[d] || c[d] >= ib->blo[d] + ib->bn[d]) ok = false;
          }
          if (!ok) continue;
          const int64_t t = (int64_t)(c[0] - ib->blo[0]) + (int64_t)(c[1] - ib->blo[1]) * ib->bn[0] +
                            (int64_t)(c[2] - ib->blo[2]) * ib->bn[0] * ib->bn[1];
          pairs.push_back({t, (m << 9) | (ii << 6) | (jj << 3) | (dim == 3 ? kk : 0)});
        }
  }
  std::stable_sort(pairs.begin(), pairs.end(),
                   [](const std::pair<int64_t, int> &x, const std::pair<int64_t, int> &y) {
                     return x.first < y.first;
                   });
  std::vector<int64_t> cells;
  std::vector<int> rowptr, ent(pairs.size());
  for (size_t e = 0; e < pairs.size(); ++e) {
    if (e == 0 || pairs[e].first != pairs[e - 1].first) {
      cells.push_back(pairs[e].first);
      rowptr.push_back((int)e);
    }
    ent[e] = pairs[e].second;
  }
  rowptr.push_back((int)pairs.size());
  const int nc = (int)cells.size();
  int rc;
  double *sw = nullptr;
  const size_t sw_doubles = (size_t)n * (sizeof(SpreadW) / sizeof(double));
  if ((rc = dmalloc(ib, &ib->d_gcell, (size_t)std::max(nc, 1))) ||
      (rc = dmalloc(ib, &ib->d_growptr, (size_t)nc + 1)) ||
      (rc = dmalloc(ib, &ib->d_gent, std::max<size_t>(ent.size(), 1))) ||
      (rc = dmalloc(ib, &sw, sw_doubles)))
    return rc;
  ib->d_sw = sw;
  cudaStream_t st = ib->ctx->stream;
  cudaError_t e = cudaMemcpyAsync(ib->d_gcell, cells.data(), nc * sizeof(int64_t), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(ib->d_growptr, rowptr.data(), (nc + 1) * sizeof(int), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && !ent.empty())
    e = cudaMemcpyAsync(ib->d_gent, ent.data(), ent.size() * sizeof(int), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_ib_create: spreading table");
  ib->gather_cells = nc;
  ib->gather = true;
  return ILBM_OK;
}

IBArgs make_args(const ilbm_ib *ib, double dt, double time) {
  IBArgs a;
  std::memset(&a, 0, sizeof(a));
  a.dim = ib->dim;
  a.kt = ib->kt;
  a.n = ib->n;
  for (int d = 0; d < 3; ++d) {
    a.plo[d] = ib->g.prob_lo[d];
    a.dx[d] = ib->dx[d];
    a.dlo[d] = 0;
    a.dhi[d] = (d < ib->dim) ? ib->g.n_cell[d] - 1 : 0;
    a.periodic[d] = (d < ib->dim) ? ib->g.periodic[d] : 0;
    a.blo[d] = ib->blo[d];
    a.bn[d] = ib->bn[d];
    a.plo_dom[d] = ib->g.prob_lo[d];
    a.phi_dom[d] = ib->g.prob_hi[d];
  }
  a.nb = ib->nb;
  a.dv = ib->dv;
  a.dt = dt;
  a.time = time;
  a.wall_tol = ib->wall_tol;
  a.geometry_type = ib->p.geometry_type;
  a.x0 = ib->p.x0;
  a.y0 = ib->p.y0;
  a.z0 = (ib->dim == 3) ? ib->p.z0 : 0.0;
  a.ub[0] = ib->p.ubx; a.ub[1] = ib->p.uby; a.ub[2] = ib->p.ubz;
  a.om[0] = ib->p.omx; a.om[1] = ib->p.omy; a.om[2] = ib->p.omz;
  a.box_yhi = ib->p.box_yhi;
  a.lid[0] = ib->p.box_lid_ux; a.lid[1] = ib->p.box_lid_uy; a.lid[2] = ib->p.box_lid_uz;
  if (ib->moving) {
    // IBMUserDefinedGeometry.H:151-160 (trigonometry on the host, in double)
    const double twopi = 2.0 * kPi;
    const double phase = twopi * ib->p.pitch_frequency * time + ib->p.pitch_phase;
    const double angle = ib->p.pitch_mean + ib->p.pitch_amplitude * std::sin(phase);
    a.komega = twopi * ib->p.pitch_frequency * ib->p.pitch_amplitude * std::cos(phase);
    a.kc = std::cos(angle);
    a.ks = std::sin(angle);
    a.pivot_x = ib->p.pivot_x;
  }
  const bool ivc = ib->p.coupling_method == 1;
  a.renorm_interp = (ib->p.renormalize_delta != 0) && !ivc;
  a.renorm_spread = (ib->p.renormalize_delta != 0);
  a.relax = std::max(0.0, std::min(1.0, ib->p.mdf_relax));
  a.diag_eps = std::max(ib->p.explicit_diag_eps, 1.0e-30);
  a.diag = (ib->p.coupling_method == 2);
  return a;
}

// storage for the explicit inverse of the fixed IVC operator (n <= ILBM_IVC_DENSE_MAX)
int enable_dense(ilbm_ib *ib) {
  if (ib->dense) return ILBM_OK;
  const int n = ib->n;
  const int ld = ((n + 31) / 32) * 32;
  int rc;
  if ((rc = dmalloc(ib, &ib->d_Ainv, (size_t)n * ld)) || (rc = dmalloc(ib, &ib->d_gj, 2 * (size_t)ld)) ||
      (rc = dmalloc(ib, &ib->d_rhs, 3 * (size_t)ld)))
    return rc;
  // the padding of the right-hand side meets zero columns of A^-1: keep it finite
  cudaError_t e = cudaMemsetAsync(ib->d_rhs, 0, 3 * (size_t)ld * sizeof(double), ib->ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "enable_dense");
  ib->ld = ld;
  ib->dense = true;
  ib->dense_ready = false;
  return ILBM_OK;
}

}  // namespace

extern "C" {

int ilbm_ib_create(ilbm_ctx *ctx, const ilbm_ib_params *p, const ilbm_level_geom *g,
                   ilbm_ib **out) {
  if (!ctx || !p || !g || !out) {
    set_error("ilbm_ib_create: null argument");
    return ILBM_ERR_ARG;
  }
  *out = nullptr;
  if (g->dim != ctx->dim) {
    set_error("ilbm_ib_create: geometry dimension differs from the lattice");
    return ILBM_ERR_ARG;
  }
  auto *ib = new ilbm_ib();
  ib->ctx = ctx;
  ib->p = *p;
  ib->g = *g;
  ib->dim = g->dim;
  ib->kt = kernel_of(p->delta_type);
  for (int d = 0; d < 3; ++d)
    ib->dx[d] = (d < g->dim) ? (g->prob_hi[d] - g->prob_lo[d]) / double(g->n_cell[d]) : 0.0;
  int rc = build_markers(ib);
  if (rc) {
    delete ib;
    return rc;
  }
  build_band(ib);
  const int n = ib->n;
  cudaSetDevice(ctx->device);
  if ((rc = dmalloc(ib, &ib->d_xyz, 3 * (size_t)n)) || (rc = dmalloc(ib, &ib->d_ref, 3 * (size_t)n)) ||
      (rc = dmalloc(ib, &ib->d_tgt, 3 * (size_t)n)) || (rc = dmalloc(ib, &ib->d_uvw, 3 * (size_t)n)) ||
      (rc = dmalloc(ib, &ib->d_F, 3 * (size_t)n)) || (rc = dmalloc(ib, &ib->d_EV, 3 * (size_t)ib->nb)) ||
      (rc = dmalloc(ib, &ib->d_EFI, 3 * (size_t)ib->nb)) || (rc = dmalloc(ib, &ib->d_EFT, 3 * (size_t)ib->nb)) ||
      (rc = dmalloc(ib, &ib->d_RHO, (size_t)ib->nb)) || (rc = dmalloc(ib, &ib->d_fsum, 4)) ||
      (rc = dmalloc(ib, &ib->d_status, 2)) || (rc = dmalloc(ib, &ib->d_iters, 2))) {
    ilbm_ib_destroy(ib);
    return rc;
  }
  std::vector<double> h(3 * (size_t)n, 0.0);
  for (int i = 0; i < n; ++i) {
    h[i] = ib->hx[i];
    h[i + n] = ib->hy[i];
    h[i + 2 * n] = ib->hz[i];
  }
  // stream-ordered like the allocations (pageable source: staged before return)
  cudaMemcpyAsync(ib->d_xyz, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
  if (!ib->xref.empty()) {
    for (int i = 0; i < n; ++i) {
      h[i] = ib->xref[i + 1];
      h[i + n] = ib->yref[i + 1];
      h[i + 2 * n] = ib->zref[i + 1];
    }
    cudaMemcpyAsync(ib->d_ref, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
  }
  cudaMemsetAsync(ib->d_status, 0, 2 * sizeof(int), ctx->stream);
  cudaMemsetAsync(ib->d_fsum, 0, 4 * sizeof(double), ctx->stream);
  // band fields finite everywhere (a fixed body forms them on its stencils only)
  cudaMemsetAsync(ib->d_EV, 0, 3 * (size_t)ib->nb * sizeof(double), ctx->stream);
  cudaMemsetAsync(ib->d_RHO, 0, (size_t)ib->nb * sizeof(double), ctx->stream);
  if ((rc = dmalloc(ib, &ib->d_recscr, force_record_scratch()))) {
    ilbm_ib_destroy(ib);
    return rc;
  }
  if ((rc = build_gather(ib))) {
    ilbm_ib_destroy(ib);
    return rc;
  }
  if (p->coupling_method == 1) {
    // neighbours per row: at most (9 cells)^d of markers within +-4 cells;
    // keep a generous cap and report overflow through the status word
    const int per_row = (ib->dim == 3) ? 512 : 96;
    ib->nnz_cap = (int)std::min<int64_t>((int64_t)n * per_row, (int64_t)n * n);
    if ((rc = dmalloc(ib, &ib->d_rowptr, (size_t)n + 1)) || (rc = dmalloc(ib, &ib->d_col, (size_t)ib->nnz_cap)) ||
        (rc = dmalloc(ib, &ib->d_val, (size_t)ib->nnz_cap)) || (rc = dmalloc(ib, &ib->d_diag, (size_t)n)) ||
        (rc = dmalloc(ib, &ib->d_X, 3 * (size_t)n)) || (rc = dmalloc(ib, &ib->d_Xh, 3 * (size_t)n)) ||
        (rc = dmalloc(ib, &ib->d_hist, 1)) ||
        (rc = dmalloc(ib, &ib->d_work, 15 * (size_t)n)) ||
        (rc = dmalloc(ib, &ib->d_tw, (size_t)kTabStride * n)) || (rc = dmalloc(ib, &ib->d_tc, (size_t)n))) {
      ilbm_ib_destroy(ib);
      return rc;
    }
    cudaMemsetAsync(ib->d_hist, 0, sizeof(int), ctx->stream);
    // grid-wide CG: as many co-resident blocks as the device holds, at most 2
    // per SM (measured fastest beside the level step it overlaps)
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ivc_cg_grid, 256, 0);
    ib->cg_blocks = std::max(1, std::min(2, per_sm) * sms);
    if ((rc = dmalloc(ib, &ib->d_partial, 16 * (size_t)std::max(per_sm * sms, 16)))) {
      ilbm_ib_destroy(ib);
      return rc;
    }
    if (!ib->moving && p->ivc_rebuild_matrix == 0 && n <= ILBM_IVC_DENSE_MAX &&
        (rc = enable_dense(ib))) {
      ilbm_ib_destroy(ib);
      return rc;
    }
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    ilbm_ib_destroy(ib);
    return cuda_fail(e, "ilbm_ib_create");
  }
  *out = ib;
  return ILBM_OK;
}

int ilbm_ib_destroy(ilbm_ib *ib) {
  if (!ib) return ILBM_OK;
  ilbm_ctx *ctx = ib->ctx;
  cudaSetDevice(ctx->device);
  // stream-ordered frees after the work queued on the context's streams
  // (the side stream's last immersed-boundary stage included): no
  // device-wide synchronisation, the memory returns to the context's pool
  cudaEventRecord(ctx->ev_fork, ctx->side);
  cudaStreamWaitEvent(ctx->stream, ctx->ev_fork, 0);
  for (void *q : ib->allocs) ilbm_ctx_free(ctx, q);
  delete ib;
  return ILBM_OK;
}

int ilbm_ib_num_markers(const ilbm_ib *ib, int64_t *n) {
  if (!ib || !n) return ILBM_ERR_ARG;
  *n = ib->n;
  return ILBM_OK;
}

int ilbm_ib_force_region(const ilbm_ib *ib, int lo[3], int hi[3]) {
  if (!ib || !lo || !hi) return ILBM_ERR_ARG;
  for (int d = 0; d < 3; ++d) {
    if (d >= ib->dim) { lo[d] = 0; hi[d] = 0; continue; }
    lo[d] = std::max(ib->blo[d], 0);
    hi[d] = std::min(ib->blo[d] + ib->bn[d] - 1, ib->g.n_cell[d] - 1);
  }
  return ILBM_OK;
}

}  // extern "C"

// Stopping tolerance of the IVC conjugate gradient (relative residual).  FP64
// populations: 1e-14, so results meet the reference's dense LU at 1e-12.
// FP32 and FP16 populations: 1e-6.  The right-hand side (U_target - U)/dt
// carries the interpolated velocity, which FP32 populations give to about
// 1e-7 absolute, 2.5e-6 relative at the sphere's U = 0.04: solving below that
// buys nothing (1e-7 costs a third iteration on the 12.9k-marker sphere and
// moves its Cd by 6e-8 relative; its Cd differs from the FP64 run's by 1e-5).
static double ivc_cg_tolerance(int storage) {
  if (storage == ILBM_STORAGE_F64) return 1.0e-14;
  return 1.0e-6;
}

// IVC solve by CG on the CSR operator (moving markers, rebuilt or large systems)
static int launch_cg(ilbm_ib *ib, const IBArgs &a_in, cudaStream_t s) {
  ilbm_ctx *ctx = ib->ctx;
  IBArgs a = a_in;
  const double cg_tol = ivc_cg_tolerance(ctx->storage);
  if (ib->n <= 1024) {
    k_ivc_cg<<<1, kCgThreads, 0, s>>>(a, ib->d_xyz, ib->d_tgt, ib->d_uvw, ib->d_rowptr, ib->d_col,
                                      ib->d_val, ib->d_diag, ib->d_X, ib->d_Xh, ib->d_hist,
                                      ib->d_work, ib->d_F, 500, cg_tol, ib->d_status, ib->d_iters);
    return ILBM_OK;
  }
  const double *xyz = ib->d_xyz, *tgt = ib->d_tgt, *uvw = ib->d_uvw, *val = ib->d_val,
               *diag = ib->d_diag;
  const int *rowptr = ib->d_rowptr, *col = ib->d_col;
  double *Xv = ib->d_X, *Xh = ib->d_Xh, *work = ib->d_work, *Fm = ib->d_F, *partial = ib->d_partial;
  int maxit = 500;
  double tol = cg_tol;
  int *hist = ib->d_hist, *status = ib->d_status, *iters = ib->d_iters;
  void *args[] = {&a, &xyz, &tgt, &uvw, &rowptr, &col, &val, &diag, &Xv, &Xh, &work, &Fm,
                  &partial, &maxit, &tol, &hist, &status, &iters};
  // one warp per ~2 rows keeps the SpMV latency-tolerant; more blocks than
  // that only make the grid barriers dearer
  const int blocks = std::max(8, std::min(ib->cg_blocks, (ib->n + 15) / 16));
  cudaError_t ce = cudaLaunchCooperativeKernel((const void *)k_ivc_cg_grid, dim3(blocks), dim3(256),
                                               args, 0, s);
  if (ce != cudaSuccess) return cuda_fail(ce, "cooperative CG launch");
  return ILBM_OK;
}

// update_forcing on stream `s` (the context stream, or its side stream when the
// chain overlaps the collide-stream of the cells outside the band)
// defer_sum: with one MDF iteration, leave the marker force sum (which only
// the force evaluation reads) to ib_finish, so it can run after the exported
// force has been handed to the level step
// boxes of a level whose grown arrays meet the body's band (or a periodic
// image of it): their StepArgs go to ib->d_boxargs (stream-ordered on s)
static int ib_box_table(ilbm_ib *ib, const ilbm_box *boxes, int nbox, const ilbm_level_params *lp,
                        cudaStream_t s) {
  ilbm_ctx *ctx = ib->ctx;
  ib->h_boxargs.clear();
  for (int b = 0; b < nbox; ++b) {
    const ilbm_box &x = boxes[b];
    if (!x.force) {
      set_error("ilbm_ib_update_forcing: every box needs its force array");
      return ILBM_ERR_ARG;
    }
    if (!x.macro_in && !x.f_in) {
      set_error("ilbm_ib_update_forcing: every box needs macro_in or f_in");
      return ILBM_ERR_ARG;
    }
    const int w = std::max(x.ngrow_f, x.ngrow_m);
    bool meets = false;
    for (int m = 0; m < 27 && !meets; ++m) {
      const int sh[3] = {m % 3 - 1, (m / 3) % 3 - 1, m / 9 - 1};
      bool ok = true, hit = true;
      for (int d = 0; d < 3; ++d) {
        if (sh[d] != 0 && (d >= ib->dim || !ib->g.periodic[d])) ok = false;
        if (d >= ib->dim) continue;
        const int lo = ib->blo[d] + sh[d] * ib->g.n_cell[d], hi = lo + ib->bn[d] - 1;
        hit = hit && hi >= x.lo[d] - w && lo <= x.hi[d] + w;
      }
      meets = ok && hit;
    }
    if (!meets) continue;
    StepArgs a;
    int rc = box_step_args(ctx, x, lp, &a);
    if (rc) return rc;
    ib->h_boxargs.push_back(a);
  }
  const int n = (int)ib->h_boxargs.size();
  if (n > ib->boxargs_cap) {
    const int cap = std::max(n, 2 * ib->boxargs_cap);
    int rc = dmalloc(ib, &ib->d_boxargs, (size_t)cap);
    if (rc) return rc;
    ib->boxargs_cap = cap;
  }
  if (n > 0) {
    cudaError_t e = cudaMemcpyAsync(ib->d_boxargs, ib->h_boxargs.data(), n * sizeof(StepArgs),
                                    cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(e, "ilbm_ib_update_forcing: box table");
  }
  return ILBM_OK;
}

static int ib_update(ilbm_ib *ib, const ilbm_box *boxes, int nbox, const ilbm_level_params *lp,
                     double dt, double time, cudaStream_t s, bool defer_sum) {
  if (!ib || !boxes || nbox < 1 || !lp) {
    set_error("ilbm_ib_update_forcing: ib, boxes (nbox >= 1) and level params are required");
    return ILBM_ERR_ARG;
  }
  ilbm_ctx *ctx = ib->ctx;
  const ilbm_box *box = boxes;
  // One box: the whole domain, or a box whose valid cells hold the body's
  // whole support band (the fine box of a two-level hierarchy), so every
  // band cell the IB reads or writes lies inside the box's arrays.  Any
  // other level takes the box-table path (caller-filled ghosts).
  bool whole = nbox == 1, holds_band = nbox == 1;
  for (int d = 0; d < ib->dim; ++d) {
    whole = whole && box->lo[d] == 0 && box->hi[d] == ib->g.n_cell[d] - 1;
    holds_band = holds_band && ib->blo[d] >= box->lo[d] && ib->blo[d] + ib->bn[d] - 1 <= box->hi[d];
  }
  const bool multi = !whole && !holds_band;
  if (multi && lp->ghost_mode != ILBM_GHOST_CALLER) {
    set_error("ilbm_ib_update_forcing: a level that is not one box holding the body's support "
              "band needs caller-filled ghosts (ILBM_GHOST_CALLER)");
    return ILBM_ERR_ARG;
  }
  for (int b = 0; b < nbox; ++b) {
    if (!boxes[b].force) {
      set_error("ilbm_ib_update_forcing: box->force is required");
      return ILBM_ERR_ARG;
    }
    if (boxes[b].macro_in && boxes[b].ngrow_m < 2) {
      set_error("ilbm_ib_update_forcing: macro_in needs at least two filled ghost layers");
      return ILBM_ERR_ARG;
    }
    if (!boxes[b].macro_in && !boxes[b].f_in) {
      set_error("ilbm_ib_update_forcing: need macro_in or f_in");
      return ILBM_ERR_ARG;
    }
  }
  const bool ivc_ = ib->p.coupling_method == 1;
  const bool single_ = ivc_ || std::max(ib->p.loop_ns, 1) == 1;
  bool periodic_band = false;
  for (int d = 0; d < ib->dim; ++d)
    periodic_band = periodic_band || (ib->g.periodic[d] && ib->blo[d] < 0);
  // EulerVel / rho on the band (:1541-1566, FillBoundary :702-703).  A body
  // whose markers do not move reads them only on the cells its stencils
  // reach (its spreading table): only those are formed.  The rest of the band
  // keeps finite values (zero at creation), which meet a zero spread force
  // in the export.
  int rc;
  if (multi) {
    if ((rc = ib_box_table(ib, boxes, nbox, lp, s))) return rc;
    rc = band_macro_boxes(ctx, ib->d_boxargs, (int)ib->h_boxargs.size(), ib->blo, ib->bn, ib->d_EV,
                          ib->d_RHO, s);
  } else if (ib->gather && single_ && !periodic_band) {
    rc = band_macro_list(ctx, *box, lp, ib->blo, ib->bn, ib->d_gcell, ib->gather_cells, ib->d_EV,
                         ib->d_RHO, s);
  } else {
    rc = band_macro(ctx, *box, lp, ib->blo, ib->bn, ib->d_EV, ib->d_RHO, s);
  }
  if (rc) return rc;
  IBArgs a = make_args(ib, dt, time);
  const int nthr = 128, nblk = (ib->n + nthr - 1) / nthr;
  const int wblk = (ib->n * 32 + 127) / 128;  // one warp per marker
  const int gb = (int)std::min<int64_t>((ib->nb + 255) / 256, 1024);
  const bool ivc = ib->p.coupling_method == 1;
  const int nloop = ivc ? 1 : std::max(ib->p.loop_ns, 1);
  const bool use_dense = ivc && ib->dense && !ib->moving && ib->p.ivc_rebuild_matrix == 0 &&
                         ib->ivc_solver != ILBM_IVC_CG;
  // with one MDF iteration the total force is the iteration's force, and the
  // velocity correction has no later reader: export straight from EFI
  const bool single = (nloop == 1);
  if (!single) cudaMemsetAsync(ib->d_EFT, 0, 3 * ib->nb * sizeof(double), s);
  cudaMemsetAsync(ib->d_fsum, 0, 3 * sizeof(double), s);
  cudaMemsetAsync(ib->d_status, 0, sizeof(int), s);
  bool any_periodic_band = false;
  for (int d = 0; d < ib->dim; ++d)
    any_periodic_band = any_periodic_band || (ib->g.periodic[d] && ib->blo[d] < 0);
  // FP64 storage (the parity form) sums interpolation and spreading in the
  // reference's order; the 4- and 2-byte forms use the warp-parallel
  // interpolation and atomic spreading, which are faster and whose rounding
  // order is far below those forms' own precision
  const bool ordered = ctx->storage == ILBM_STORAGE_F64;
  // markers that do not move: their kernel weights once, for the ordered
  // spreading (FP64) or the table-driven interpolation and spreading
  SpreadW *sw = static_cast<SpreadW *>(ib->d_sw);
  if (ib->gather && !ib->sw_ready) {
    k_spread_weights<<<nblk, nthr, 0, s>>>(a, ib->d_xyz, sw);
    ctx->launches++;
    ib->sw_ready = true;
  }
  const bool table = ib->gather && !ordered;
  // the warp-parallel interpolation (k_interp) writes the step's weight table
  // of an IVC body, which its operator build and spreading then read
  double *tw = (!ordered && !table) ? ib->d_tw : nullptr;
  int4 *tc = tw ? ib->d_tc : nullptr;
  for (int it = 0; it < nloop; ++it) {
    cudaMemsetAsync(ib->d_EFI, 0, 3 * ib->nb * sizeof(double), s);
    // a fixed body's markers need no position update: the table-driven
    // interpolation zeroes their velocities and forces itself
    const bool fresh = table && ib->p.geometry_type != 2;
    if (!fresh) k_markers<<<nblk, nthr, 0, s>>>(a, ib->d_xyz, ib->d_ref, ib->d_tgt, ib->d_uvw, ib->d_F);
    if (any_periodic_band) k_fill_boundary<<<gb, 256, 0, s>>>(a, ib->d_EV);
    if (ordered)
      k_interp_seq<<<nblk, nthr, 0, s>>>(a, ib->d_xyz, ib->d_EV, ib->d_uvw, ib->d_status, ib->d_tgt,
                                         use_dense ? ib->d_rhs : nullptr, ib->ld);
    else if (table)
      k_interp_w<<<wblk, 128, 0, s>>>(a, ib->d_xyz, sw, ib->d_EV, ib->d_uvw, ib->d_F, fresh ? 1 : 0,
                                      ib->d_status, ib->d_tgt, use_dense ? ib->d_rhs : nullptr, ib->ld);
    else
      k_interp<<<wblk, 128, 0, s>>>(a, ib->d_xyz, ib->d_EV, ib->d_uvw, ib->d_status, ib->d_tgt,
                                    use_dense ? ib->d_rhs : nullptr, ib->ld, tw, tc);
    ctx->launches += (fresh ? 1 : 2) + (any_periodic_band ? 1 : 0);
    if (ivc) {
      if (!ib->csr_ready || ib->moving || ib->p.ivc_rebuild_matrix > 0) {
        const int cb = std::min(4096, (ib->n * 32 + 255) / 256);
        k_csr_count<<<cb, 256, 0, s>>>(a, ib->d_xyz, ib->d_rowptr, tc);
        k_csr_scan<<<1, 1024, 0, s>>>(ib->n, ib->d_rowptr, ib->nnz_cap, ib->d_status);
        k_csr_fill<<<cb, 256, 0, s>>>(a, ib->d_xyz, ib->p.ivc_diag_reg, ib->d_rowptr, ib->d_col,
                                      ib->d_val, ib->d_diag, ib->nnz_cap, ib->d_status, tw, tc);
        ctx->launches += 3;
        ib->csr_ready = true;
      }
      if (use_dense) {
        if (!ib->dense_ready) {
          // once per body: dense copy of the operator, then Gauss-Jordan in place
          const int n = ib->n, ld = ib->ld;
          const int cb = std::min(4096, (n * 32 + 255) / 256);
          double *rowk = ib->d_gj, *colk = ib->d_gj + ld;
          cudaMemsetAsync(ib->d_Ainv, 0, (size_t)n * ld * sizeof(double), s);
          cudaMemsetAsync(ib->d_iters, 0, sizeof(int), s);
          k_dense_scatter<<<cb, 256, 0, s>>>(n, ld, ib->d_rowptr, ib->d_col, ib->d_val, ib->d_Ainv);
          const int pb = (n + 255) / 256;
          for (int k = 0; k < n; ++k) {
            k_gj_panel<<<pb, 256, 0, s>>>(ib->d_Ainv, n, ld, k, rowk, colk, ib->d_status);
            k_gj_update<<<n, 256, 0, s>>>(ib->d_Ainv, n, ld, k, rowk, colk, ib->d_status);
          }
          ctx->launches += 1 + 2 * (int64_t)n;
          if (ctx->storage != ILBM_STORAGE_F64) {
            if (!ib->d_Ainv32 && (rc = dmalloc(ib, &ib->d_Ainv32, (size_t)n * ld))) return rc;
            k_to_f32<<<1024, 256, 0, s>>>(ib->d_Ainv, ib->d_Ainv32, (int64_t)n * ld);
            ctx->launches++;
          }
          ib->dense_ready = true;
        }
        const int db = (ib->n + kDenseRows - 1) / kDenseRows;
        if (ib->d_Ainv32)
          k_ivc_dense_rows<float><<<db, kDenseThreads, 0, s>>>(a, ib->d_rhs, ib->d_Ainv32, ib->ld, ib->d_F);
        else
          k_ivc_dense_rows<double><<<db, kDenseThreads, 0, s>>>(a, ib->d_rhs, ib->d_Ainv, ib->ld, ib->d_F);
      } else if ((rc = launch_cg(ib, a, s))) {
        return rc;
      }
      ctx->launches++;
    } else {
      k_force_explicit<<<nblk, nthr, 0, s>>>(a, ib->d_xyz, ib->d_tgt, ib->d_uvw, ib->d_F);
      ctx->launches++;
    }
    if (ordered && ib->gather) {
      k_spread_gather<<<(ib->gather_cells + 127) / 128, 128, 0, s>>>(
          a, sw, ib->d_F, ib->d_gcell, ib->d_growptr, ib->d_gent, ib->gather_cells, ib->d_EFI);
      ctx->launches++;
    } else if (table) {
      k_spread_w<<<wblk, 128, 0, s>>>(a, ib->d_xyz, sw, ib->d_F, ib->d_EFI, ib->d_status);
      ctx->launches++;
    } else {
      k_spread<<<wblk, 128, 0, s>>>(a, ib->d_xyz, ib->d_F, ib->d_EFI, ib->d_status, tw, tc);
      ctx->launches++;
    }
    if (any_periodic_band) {
      k_sum_boundary<<<gb, 256, 0, s>>>(a, ib->d_EFI);
      ctx->launches++;
    }
    ib->fsum_deferred = single && defer_sum;
    if (!ib->fsum_deferred) {
      k_marker_sum<<<1, 1024, 0, s>>>(a, ib->d_F, ib->d_fsum);
      ctx->launches++;
    }
    if (!single) {
      k_correct<<<gb, 256, 0, s>>>(a, ib->d_EV, ib->d_EFI, ib->d_EFT);
      ctx->launches++;
    }
  }
  const double *EFT = single ? ib->d_EFI : ib->d_EFT;
  const int mgl0 = box->lo[0] - box->ngrow_m, mgl1 = box->lo[1] - box->ngrow_m;
  const int mgl2 = (ib->dim == 3) ? box->lo[2] - box->ngrow_m : 0;
  if (multi) {
    const int nargs = (int)ib->h_boxargs.size();
    if (ctx->storage == ILBM_STORAGE_F64)
      k_export_boxes<double><<<gb, 256, 0, s>>>(a, EFT, ib->d_RHO, ib->d_boxargs, nargs);
    else
      k_export_boxes<float><<<gb, 256, 0, s>>>(a, EFT, ib->d_RHO, ib->d_boxargs, nargs);
  } else if (ctx->storage == ILBM_STORAGE_F64)
    k_export<double><<<gb, 256, 0, s>>>(a, EFT, ib->d_RHO, static_cast<double *>(box->force),
                                        mgl0, mgl1, mgl2, box->mstride[0], box->mstride[1], box->mstride[2]);
  else
    k_export<float><<<gb, 256, 0, s>>>(a, EFT, ib->d_RHO, static_cast<float *>(box->force),
                                       mgl0, mgl1, mgl2, box->mstride[0], box->mstride[1], box->mstride[2]);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_ib_update_forcing");
  return ILBM_OK;
}

// the work ib_update deferred (the marker force sum), on stream s
static int ib_finish(ilbm_ib *ib, cudaStream_t s) {
  if (!ib->fsum_deferred) return ILBM_OK;
  k_marker_sum<<<1, 1024, 0, s>>>(make_args(ib, 1.0, 0.0), ib->d_F, ib->d_fsum);
  ib->ctx->launches++;
  ib->fsum_deferred = false;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "marker force sum");
  return ILBM_OK;
}

namespace ilbm {

int advance_begin(ilbm_ctx *ctx, const ilbm_box *box, const ilbm_level_params *p, ilbm_ib *ib,
                  double dt, double time, AdvanceSplit *sp) {
  if (ib->ctx != ctx) {
    set_error("ilbm_advance_level: the IB object belongs to another context");
    return ILBM_ERR_ARG;
  }
  sp->q = *p;
  ilbm_ib_force_region(ib, sp->lo, sp->hi);
  for (int d = 0; d < 3; ++d) {
    sp->q.force_lo[d] = sp->lo[d];
    sp->q.force_hi[d] = sp->hi[d];
  }
  // caller-filled ghosts covered by other boxes of the level may carry their
  // IB forces, so those levels run serially; one box that holds the whole
  // band (the fine box of a two-level hierarchy) overlaps like self-fill
  bool band_inside = p->nlevel_boxes <= 1 && box->f_in != box->f_out;
  for (int d = 0; d < ctx->dim; ++d)
    band_inside = band_inside && sp->lo[d] >= box->lo[d] && sp->hi[d] <= box->hi[d];
  sp->serial = (p->ghost_mode != ILBM_GHOST_SELF && !band_inside);
  if (sp->serial) return ib_update(ib, box, 1, &sp->q, dt, time, ctx->stream, false);
  // validate like ilbm_level_step does before anything is launched
  if ((p->ghost_mode == ILBM_GHOST_SELF && box->lo[0] != p->domain_lo[0]) || box->f_in == box->f_out) {
    set_error("ilbm_advance_level: self-fill needs one box equal to the domain, f_in != f_out");
    return ILBM_ERR_ARG;
  }
  // the IB chain runs on the side stream, after what the main stream holds so
  // far, while the main stream goes on with other work
  cudaError_t e = cudaEventRecord(ctx->ev_fork, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->side, ctx->ev_fork, 0);
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_advance_level fork");
  int rc = ib_update(ib, box, 1, &sp->q, dt, time, ctx->side, true);
  if (rc) return rc;
  e = cudaEventRecord(ctx->ev_join, ctx->side);
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_advance_level join");
  // the marker force sum runs beside the band's collide-stream
  if ((rc = ib_finish(ib, ctx->side))) return rc;
  e = cudaEventRecord(ctx->ev_done, ctx->side);
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_advance_level done");
  return ILBM_OK;
}

int advance_end(ilbm_ctx *ctx, const ilbm_box *box, const AdvanceSplit *sp) {
  if (sp->serial) return ilbm_level_step(ctx, box, 1, &sp->q);
  // the collide-stream of every cell outside the band, then the band once
  // the body's forcing is in
  int rc = level_step_split(ctx, *box, &sp->q, sp->lo, sp->hi, ctx->ev_join);
  if (rc) return rc;
  cudaError_t e = cudaStreamWaitEvent(ctx->stream, ctx->ev_done, 0);
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_advance_level wait");
  return ILBM_OK;
}

}  // namespace ilbm

extern "C" {

int ilbm_ib_update_forcing(ilbm_ib *ib, const ilbm_box *boxes, int nbox,
                           const ilbm_level_params *lp, double dt, double time) {
  if (!ib) {
    set_error("ilbm_ib_update_forcing: null ib");
    return ILBM_ERR_ARG;
  }
  return ib_update(ib, boxes, nbox, lp, dt, time, ib->ctx->stream, false);
}

int ilbm_advance_level(ilbm_ctx *ctx, const ilbm_box *box, const ilbm_level_params *p,
                       ilbm_ib *ib, double dt, double time) {
  if (!ctx || !box || !p) {
    set_error("ilbm_advance_level: null argument");
    return ILBM_ERR_ARG;
  }
  if (!ib) return ilbm_level_step(ctx, box, 1, p);
  AdvanceSplit sp;
  int rc = advance_begin(ctx, box, p, ib, dt, time, &sp);
  if (rc) return rc;
  return advance_end(ctx, box, &sp);
}

int ilbm_ib_last_marker_force_sum(ilbm_ib *ib, double out[3]) {
  if (!ib || !out) return ILBM_ERR_ARG;
  ilbm_ctx *ctx = ib->ctx;
  int st[2] = {0, 0};
  cudaMemcpyAsync(ctx->host_pinned, ib->d_fsum, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemcpyAsync(st, ib->d_status, 2 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "marker force sum");
  for (int c = 0; c < 3; ++c) out[c] = ctx->host_pinned[c];
  if (st[0] & 1) {
    set_error("IB stencil left the support band (marker outside its envelope)");
    return ILBM_ERR_RANGE;
  }
  if (st[0] & 2) {
    set_error("IVC operator exceeded its nonzero capacity");
    return ILBM_ERR_SOLVER;
  }
  if (st[0] & 4) {
    set_error("IVC conjugate gradient did not converge");
    return ILBM_ERR_SOLVER;
  }
  if (st[1] & 8) {
    set_error("IVC operator has a non-positive pivot (not positive definite); its inverse is invalid");
    return ILBM_ERR_SOLVER;
  }
  return ILBM_OK;
}

}  // extern "C"

int ilbm::ib_record_on(ilbm_ib *ib, const ilbm_box &box, const int lo[3], const int hi[3],
                       double *rec, cudaStream_t st) {
  ilbm_ctx *ctx = ib->ctx;
  int rc = force_record_on(ctx, box, lo, hi, ib->d_fsum, ib->d_status, rec, ib->d_recscr, st);
  if (rc) return rc;
  cudaError_t e = cudaEventRecord(ctx->ev_rec, st);
  if (e != cudaSuccess) return cuda_fail(e, "force record event");
  return ILBM_OK;
}

extern "C" {

int ilbm_force_record_async(ilbm_ctx *ctx, const ilbm_box *boxes, int nbox, ilbm_ib *ib,
                            const int lo[3], const int hi[3], double *out) {
  if (!ctx || !boxes || nbox < 1 || !ib || !out) {
    set_error("ilbm_force_record_async: null argument");
    return ILBM_ERR_ARG;
  }
  if (ib->ctx != ctx) {
    set_error("ilbm_force_record_async: the IB object belongs to another context");
    return ILBM_ERR_ARG;
  }
  // the sums' final launch also packs the record: straight into `out` when it
  // is pinned host memory the device can address (no copy on the stream),
  // else into scratch, copied to `out` after it
  double *direct = nullptr;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, out) == cudaSuccess) {
    if (at.type == cudaMemoryTypeHost && at.devicePointer)
      direct = static_cast<double *>(at.devicePointer);
    else if (at.type == cudaMemoryTypeDevice && at.device == ctx->device)
      direct = out;
  }
  cudaGetLastError();  // an unregistered pointer is not an error here
  double *d_sum = nullptr;
  int rc = force_sum_enqueue(ctx, boxes, nbox, lo, hi, &d_sum, ib->d_fsum, ib->d_status, direct);
  if (rc) return rc;
  if (direct) return ILBM_OK;
  cudaError_t e = cudaMemcpyAsync(out, d_sum + 8, 8 * sizeof(double), cudaMemcpyDefault, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_force_record_async");
  return ILBM_OK;
}

int ilbm_ib_solver_stats(ilbm_ib *ib, int *cg_iterations) {
  if (!ib || !cg_iterations) return ILBM_ERR_ARG;
  int it = 0;
  cudaMemcpyAsync(&it, ib->d_iters, sizeof(int), cudaMemcpyDeviceToHost, ib->ctx->stream);
  cudaError_t e = cudaStreamSynchronize(ib->ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_ib_solver_stats");
  *cg_iterations = (ib->p.coupling_method == 1) ? it : 0;
  return ILBM_OK;
}

int ilbm_ib_set_ivc_solver(ilbm_ib *ib, int solver) {
  if (!ib || solver < ILBM_IVC_AUTO || solver > ILBM_IVC_DENSE) {
    set_error("ilbm_ib_set_ivc_solver: bad argument");
    return ILBM_ERR_ARG;
  }
  if (solver == ILBM_IVC_DENSE) {
    if (ib->p.coupling_method != 1 || ib->moving || ib->p.ivc_rebuild_matrix > 0 ||
        ib->n > ILBM_IVC_DENSE_MAX) {
      set_error("ilbm_ib_set_ivc_solver: the stored inverse needs implicit velocity correction, "
                "fixed markers, no matrix rebuild and at most ILBM_IVC_DENSE_MAX markers");
      return ILBM_ERR_UNSUPPORTED;
    }
    cudaSetDevice(ib->ctx->device);
    const int rc = enable_dense(ib);
    if (rc) return rc;
  }
  ib->ivc_solver = solver;
  if (ib->d_hist) {  // the next solve starts from zero
    cudaError_t e = cudaMemsetAsync(ib->d_hist, 0, sizeof(int), ib->ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "ilbm_ib_set_ivc_solver");
  }
  return ILBM_OK;
}

int ilbm_ib_markers(ilbm_ib *ib, double *xyz, double *uvw, double *force) {
  if (!ib) return ILBM_ERR_ARG;
  ilbm_ctx *ctx = ib->ctx;
  const size_t nbytes = 3 * (size_t)ib->n * sizeof(double);
  if (xyz) cudaMemcpyAsync(xyz, ib->d_xyz, nbytes, cudaMemcpyDeviceToHost, ctx->stream);
  if (uvw) cudaMemcpyAsync(uvw, ib->d_uvw, nbytes, cudaMemcpyDeviceToHost, ctx->stream);
  if (force) cudaMemcpyAsync(force, ib->d_F, nbytes, cudaMemcpyDeviceToHost, ctx->stream);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_ib_markers");
  return ILBM_OK;
}

}  // extern "C"

namespace ilbm {

void ib_state(ilbm_ib *ib, IBState *out) {
  out->n = ib->n;
  out->dim = ib->dim;
  out->geometry = ib->p.geometry_type;
  out->coupling = ib->p.coupling_method;
  out->xyz = ib->d_xyz;
  out->uvw = ib->d_uvw;
  out->F = ib->d_F;
  out->fsum = ib->d_fsum;
  out->X = ib->d_X;
  out->Xh = ib->d_Xh;
  // the solves keep the history count on the device (the caller has
  // synchronised the context's stream)
  int h = 0;
  if (ib->d_hist && cudaMemcpy(&h, ib->d_hist, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    h = 0;
  out->cg_warm = h >= 1;
  out->cg_hist2 = h >= 2;
}

void ib_set_cg_warm(ilbm_ib *ib, bool warm, bool hist2) {
  if (!ib->d_hist) return;
  const int h = (warm && ib->d_X) ? ((hist2 && ib->d_Xh) ? 2 : 1) : 0;
  cudaMemcpy(ib->d_hist, &h, sizeof(int), cudaMemcpyHostToDevice);
}

}  // namespace ilbm


// ---------------------------------------------------------------------------
// Batched update_forcing for the batch engine (batch.cu): every stage runs as
// one launch over all cases.  The items of a stage (markers, band tiles, rows
// of a stored inverse) come from work lists of (case, item) built when the
// batch is formed; each case's IBArgs and arrays sit in a device table, and
// the operator build runs over the markers of rebuilding bodies only.  Cases have
// taken their first step through ib_update already (operator and inverse
// built), use one MDF iteration, and read the time-dependent pitching
// kinematics from a per-step table filled on the host with the same
// arithmetic as make_args.
// ---------------------------------------------------------------------------

namespace {

struct IBCase {
  IBArgs a;
  double *xyz;
  const double *ref;
  double *tgt, *uvw, *F, *EV, *EFI, *RHO, *fsum;
  int *status, *iters;
  int mode;     // 0 explicit, 1 stored inverse, 2 CG
  int rebuild;  // CG operator rebuilt every step (moving markers / ivc_rebuild_matrix)
  int moving, periodic_band;
  int *rowptr, *col;
  double *val, *diag, *X, *Xh, *work;
  int *hist;
  int nnz_cap;
  double reg, cg_tol;
  const double *Ainv;
  const float *Ainv32;  // used instead of Ainv when set
  double *rhs;
  int ld;
  const double *kin;  // per step: komega, cos, sin, 0
  int kin_steps;
  double *rec;        // rec_slots x 8: Eulerian force sum (3), marker force sum (3), step, 0
  double *tw;         // the step's marker weight table (kTabStride per marker) and cells
  int4 *tc;
  int tile0, ntile;   // the case's band tiles in the batch's tile list
};

// a case that has taken all the steps it was added for sits out
__device__ __forceinline__ bool live(const int *steps, const int *limit, int c) {
  return steps[c] < limit[c];
}

__global__ void __launch_bounds__(256) k_b_markers(const IBCase *cs, const ItemRef *list, int64_t cnt,
                                                   const int *steps, const int *limit) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < cnt;
       t += (int64_t)gridDim.x * blockDim.x) {
    const ItemRef e = list[t];
    const int c = e.c;
    if (!live(steps, limit, c)) continue;
    const IBCase &k = cs[c];
    const int m = e.u;
    if (m == 0) {
      k.fsum[0] = k.fsum[1] = k.fsum[2] = 0.0;
      k.status[0] = 0;
    }
    double kc = 1.0, ks = 0.0, om = 0.0;
    if (k.moving) {
      int s = steps[c];
      if (s >= k.kin_steps) {
        if (m == 0) atomicOr(k.status, 16);  // ran past its kinematics table
        s = k.kin_steps - 1;
      }
      om = k.kin[4 * s];
      kc = k.kin[4 * s + 1];
      ks = k.kin[4 * s + 2];
    }
    markers_one(k.a, kc, ks, om, m, k.xyz, k.ref, k.tgt, k.uvw, k.F);
  }
}

// one block of kItemTile threads per band tile
__global__ void __launch_bounds__(kItemTile) k_b_band(const IBCase *cs, const ItemRef *tiles, int ntiles,
                                                      int op, const int *steps, const int *limit) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const ItemRef e = tiles[t];
    const int c = e.c;
    if (!live(steps, limit, c)) continue;
    const IBCase &k = cs[c];
    const int64_t u = (int64_t)e.u + threadIdx.x;
    if (u >= k.a.nb) continue;
    if (op == 0) {
      k.EFI[u] = 0.0;
      k.EFI[u + k.a.nb] = 0.0;
      k.EFI[u + 2 * k.a.nb] = 0.0;
    } else if (op == 1) {
      if (k.periodic_band) fill_boundary_cell(k.a, k.EV, u);
    } else {
      if (k.periodic_band) sum_boundary_cell(k.a, k.EFI, u);
    }
  }
}

// one warp per marker; stage 0 interpolation (writes the weight table), 1
// explicit force, 2 spreading, 3 CSR row count, 4 CSR row fill (2-4 read the
// table)
template <int stage>
__global__ void __launch_bounds__(128) k_b_marker_warp(const IBCase *cs, const ItemRef *list, int64_t cnt,
                                                       const int *steps, const int *limit) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < cnt; w += nw) {
    const ItemRef e = list[w];
    const int c = e.c;
    if (!live(steps, limit, c)) continue;
    const IBCase &k = cs[c];
    const int m = e.u;
    if constexpr (stage == 0) {
      interp_one(k.a, m, lane, k.xyz, k.EV, k.uvw, k.status, k.tgt, k.mode == 1 ? k.rhs : nullptr,
                 k.ld, k.tw, k.tc);
    } else if constexpr (stage == 1) {
      if (k.mode == 0 && lane == 0) force_explicit_one(k.a, m, k.xyz, k.tgt, k.uvw, k.F);
    } else if constexpr (stage == 2) {
      spread_one_tab(k.a, m, lane, k.tw, k.tc, k.F, k.EFI, k.status);
    } else if constexpr (stage == 3) {
      if (k.mode == 2 && k.rebuild) csr_count_row(k.a, k.xyz, k.rowptr, m, lane, k.tc);
    } else {
      if (k.mode == 2 && k.rebuild && !(k.status[0] & 2) && k.rowptr[k.a.n] <= k.nnz_cap)
        csr_fill_row(k.a, k.xyz, k.reg, k.rowptr, k.col, k.val, k.diag, m, lane, k.tw, k.tc);
    }
  }
}

// one block per CG case: the CSR scan of a rebuilding body
__global__ void __launch_bounds__(kCgThreads) k_b_scan(const IBCase *cs, const int *cg_case,
                                                 const int *steps, const int *limit) {
  if (!live(steps, limit, cg_case[blockIdx.x])) return;
  const IBCase &k = cs[cg_case[blockIdx.x]];
  if (k.rebuild) csr_scan_block(k.a.n, k.rowptr, k.nnz_cap, k.status);
}

// one block per CG case: the solve
__global__ void __launch_bounds__(kCgThreads) k_b_cg(const IBCase *cs, const int *cg_case,
                                                     const int *steps, const int *limit) {
  __shared__ double p_sh[3 * kCgSharedN];
  if (!live(steps, limit, cg_case[blockIdx.x])) return;
  const IBCase &k = cs[cg_case[blockIdx.x]];
  ivc_cg_block(k.a, k.xyz, k.tgt, k.uvw, k.rowptr, k.col, k.val, k.diag, k.X, k.Xh, k.hist, k.work,
               k.F, 500, k.cg_tol, k.status, k.iters, p_sh);
}

// one block per row of every stored inverse (list: case, row)
__global__ void __launch_bounds__(kDenseThreads) k_b_dense(const IBCase *cs, const ItemRef *rows,
                                                           const int *steps, const int *limit) {
  const ItemRef e = rows[blockIdx.x];
  if (!live(steps, limit, e.c)) return;
  const IBCase &k = cs[e.c];
  if (k.Ainv32)
    dense_row32(k.a, k.rhs, k.Ainv32, k.ld, k.F, e.u);
  else
    dense_row(k.a, k.rhs, k.Ainv, k.ld, k.F, e.u);
}

template <class R>
// each tile also leaves the fixed-order sum of the force it stored (tpart,
// 3 per tile): the case's Eulerian force sum, combined by k_b_record
__global__ void __launch_bounds__(kItemTile) k_b_export(const IBCase *cs, const ItemRef *tiles,
                                                        int ntiles, const StepArgs *args,
                                                        const int *steps, const int *limit,
                                                        double *tpart) {
  __shared__ double shr[kMaxWarps][3];
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const ItemRef e = tiles[t];
    const int c = e.c;
    if (!live(steps, limit, c)) continue;  // uniform over the block
    const IBCase &k = cs[c];
    const int64_t u = (int64_t)e.u + threadIdx.x;
    double v[3] = {0.0, 0.0, 0.0};
    if (u < k.a.nb) {
      const StepArgs &sa = args[c];
      export_cell<R>(k.a, k.EFI, k.RHO, static_cast<R *>(const_cast<void *>(sa.force)), sa.mgl[0],
                     sa.mgl[1], sa.mgl[2], sa.ms0, sa.ms1, sa.ms2, u, v);
    }
    double tot[3];
    block_reduce<3>(v, shr, tot);
    if (threadIdx.x == 0) {
      tpart[3 * (int64_t)t] = tot[0];
      tpart[3 * (int64_t)t + 1] = tot[1];
      tpart[3 * (int64_t)t + 2] = tot[2];
    }
    __syncthreads();  // shr is read before the next tile's reduction writes it
  }
}

// one block per case: its Eulerian force sum (the export's tile partials in
// tile order), the marker force sum, a record ring entry and the step counter
constexpr int kRecThreads = 256;
__global__ void __launch_bounds__(kRecThreads) k_b_record(const IBCase *cs, int *steps,
                                                          const int *limit, int rec_slots,
                                                          const double *tpart) {
  __shared__ double sh[33];
  const int c = blockIdx.x;
  if (!live(steps, limit, c)) return;
  const IBCase &k = cs[c];
  double fe[3] = {0.0, 0.0, 0.0};
  if (k.a.n > 0) {
    marker_sum_block(k.a, k.F, k.fsum);
    for (int comp = 0; comp < 3; ++comp) {
      double sm = 0.0;
      for (int q = threadIdx.x; q < k.ntile; q += blockDim.x)
        sm += tpart[3 * (int64_t)(k.tile0 + q) + comp];
      fe[comp] = block_sum(sm, sh);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int st = steps[c];
    double *r = k.rec + (size_t)(st % rec_slots) * 8;
    r[0] = fe[0];
    r[1] = fe[1];
    r[2] = fe[2];
    r[3] = (k.a.n > 0) ? k.fsum[0] : 0.0;
    r[4] = (k.a.n > 0) ? k.fsum[1] : 0.0;
    r[5] = (k.a.n > 0) ? k.fsum[2] : 0.0;
    r[6] = double(st);
    r[7] = 0.0;
    steps[c] = st + 1;
  }
}

}  // namespace

namespace ilbm {

struct IBBatch {
  ilbm_ctx *ctx = nullptr;
  int nc = 0, rec_slots = 1;
  std::vector<void *> allocs;
  IBCase *d_cases = nullptr;
  BandDesc *d_bands = nullptr;
  int64_t total_m = 0, total_b = 0, total_drows = 0, total_rm = 0;
  int nbt = 0;  // band tiles
  // work lists: every marker, the markers of bodies whose operator is
  // rebuilt each step, every row of a stored inverse (case, item), and the
  // band tiles (case, first cell)
  ItemRef *d_mlist = nullptr, *d_rlist = nullptr, *d_dlist = nullptr, *d_btiles = nullptr;
  int *d_cgcase = nullptr;
  int ncg = 0;
  bool any_periodic = false, any_explicit = false, any_rebuild = false;
  int *d_steps = nullptr, *d_limit = nullptr;
  double *d_rec = nullptr, *d_tpart = nullptr;  // record rings; the export's tile partials
  // fork / join of the moving bodies' operator build and CG (on the context's
  // high-priority side stream) beside the stored-inverse solves
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  int *d_status_copy = nullptr;
  std::vector<int *> status_ptrs;
};

template <class T>
static int bmalloc(IBBatch *b, T **p, size_t count) {
  void *q = nullptr;
  cudaError_t e = ilbm_ctx_malloc(b->ctx, &q, count * sizeof(T));
  if (e != cudaSuccess) return cuda_fail(e, "device allocation (IB batch)");
  b->allocs.push_back(q);
  *p = static_cast<T *>(q);
  return ILBM_OK;
}
template <class T>
static int bupload(IBBatch *b, T **p, const std::vector<T> &h) {
  int rc = bmalloc(b, p, std::max<size_t>(1, h.size()));
  if (rc) return rc;
  if (!h.empty()) {
    cudaError_t e = cudaMemcpyAsync(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice,
                                    b->ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "IB batch upload");
  }
  return ILBM_OK;
}
static int grid_for(int64_t items, int threads) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((items + threads - 1) / threads, 4096));
}

void ib_batch_destroy(IBBatch *b) {
  if (!b) return;
  // (the side stream's batch work joined the context's stream before any
  // later work there: the frees are ordered after it)
  for (void *q : b->allocs) ilbm_ctx_free(b->ctx, q);
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  if (b->ev_join) cudaEventDestroy(b->ev_join);
  delete b;
}

int ib_batch_create(ilbm_ctx *ctx, const std::vector<IBBatchCase> &cases, int rec_slots,
                    IBBatch **out) {
  *out = nullptr;
  auto *b = new IBBatch();
  b->ctx = ctx;
  {
    cudaError_t e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming);
    if (e != cudaSuccess) {
      ib_batch_destroy(b);
      return cuda_fail(e, "IB batch events");
    }
  }
  b->nc = (int)cases.size();
  b->rec_slots = std::max(1, rec_slots);
  std::vector<IBCase> hc(b->nc);
  std::vector<BandDesc> hb(b->nc);
  std::vector<int64_t> moff(b->nc + 1, 0), boff(b->nc + 1, 0);
  std::vector<int> cgcase;
  std::vector<ItemRef> mlist, rlist, dlist, btiles;
  std::vector<std::vector<double>> kin(b->nc);
  for (int c = 0; c < b->nc; ++c) {
    IBCase &k = hc[c];
    std::memset(&k, 0, sizeof(k));
    BandDesc &bd = hb[c];
    std::memset(&bd, 0, sizeof(bd));
    ilbm_ib *ib = cases[c].ib;
    moff[c + 1] = moff[c];
    boff[c + 1] = boff[c];
    b->status_ptrs.push_back(nullptr);
    if (!ib) continue;
    if (ib->ctx != ctx) {
      set_error("batch: an IB object belongs to another context");
      ib_batch_destroy(b);
      return ILBM_ERR_ARG;
    }
    const bool ivc = ib->p.coupling_method == 1;
    if (!ivc && ib->p.loop_ns > 1) {
      set_error("batch: explicit coupling with several MDF iterations (loop_ns > 1) is not batched");
      ib_batch_destroy(b);
      return ILBM_ERR_UNSUPPORTED;
    }
    if (ivc && !ib->csr_ready) {
      set_error("batch: a body joins after its first step (its IVC operator is not built yet)");
      ib_batch_destroy(b);
      return ILBM_ERR_ARG;
    }
    k.a = make_args(ib, cases[c].dt, cases[c].time0);
    k.xyz = ib->d_xyz;
    k.ref = ib->d_ref;
    k.tgt = ib->d_tgt;
    k.uvw = ib->d_uvw;
    k.F = ib->d_F;
    k.EV = ib->d_EV;
    k.EFI = ib->d_EFI;
    k.RHO = ib->d_RHO;
    k.fsum = ib->d_fsum;
    k.status = ib->d_status;
    k.iters = ib->d_iters;
    k.moving = ib->moving ? 1 : 0;
    for (int d = 0; d < ib->dim; ++d)
      k.periodic_band = k.periodic_band || (ib->g.periodic[d] && ib->blo[d] < 0);
    const bool dense = ivc && ib->dense && ib->dense_ready && !ib->moving &&
                       ib->p.ivc_rebuild_matrix == 0 && ib->ivc_solver != ILBM_IVC_CG;
    k.mode = !ivc ? 0 : (dense ? 1 : 2);
    k.rebuild = (k.mode == 2 && (ib->moving || ib->p.ivc_rebuild_matrix > 0)) ? 1 : 0;
    k.rowptr = ib->d_rowptr;
    k.col = ib->d_col;
    k.val = ib->d_val;
    k.diag = ib->d_diag;
    k.X = ib->d_X;
    k.Xh = ib->d_Xh;
    k.hist = ib->d_hist;
    k.work = ib->d_work;
    k.nnz_cap = ib->nnz_cap;
    k.reg = ib->p.ivc_diag_reg;
    k.cg_tol = ivc_cg_tolerance(ctx->storage);
    k.Ainv = ib->d_Ainv;
    k.Ainv32 = ib->d_Ainv32;
    k.rhs = ib->d_rhs;
    k.ld = ib->ld;
    if (ib->moving) {
      // IBMUserDefinedGeometry.H:151-160 with the time accumulated step by
      // step as the caller does (time += dt), host trigonometry as make_args
      const int ns = std::max(1, cases[c].kin_steps);
      kin[c].assign(4 * (size_t)ns, 0.0);
      double t = cases[c].time0;
      const double twopi = 2.0 * kPi;
      for (int s = 0; s < ns; ++s) {
        const double phase = twopi * ib->p.pitch_frequency * t + ib->p.pitch_phase;
        const double angle = ib->p.pitch_mean + ib->p.pitch_amplitude * std::sin(phase);
        kin[c][4 * s] = twopi * ib->p.pitch_frequency * ib->p.pitch_amplitude * std::cos(phase);
        kin[c][4 * s + 1] = std::cos(angle);
        kin[c][4 * s + 2] = std::sin(angle);
        t += cases[c].dt;
      }
      k.kin_steps = ns;
    }
    moff[c + 1] = moff[c] + ib->n;
    boff[c + 1] = boff[c] + ib->nb;
    for (int m = 0; m < ib->n; ++m) {
      mlist.push_back({c, m});
      if (k.rebuild) rlist.push_back({c, m});
      if (k.mode == 1) dlist.push_back({c, m});
    }
    k.tile0 = (int)btiles.size();
    for (int64_t u = 0; u < ib->nb; u += kItemTile) btiles.push_back({c, (int)u});
    k.ntile = (int)btiles.size() - k.tile0;
    for (int d = 0; d < 3; ++d) {
      bd.blo[d] = ib->blo[d];
      bd.bn[d] = ib->bn[d];
    }
    bd.nb = ib->nb;
    bd.EV = ib->d_EV;
    bd.RHO = ib->d_RHO;
    bd.EFI = ib->d_EFI;
    if (k.mode == 2) cgcase.push_back(c);
    b->any_periodic = b->any_periodic || k.periodic_band;
    b->any_explicit = b->any_explicit || k.mode == 0;
    b->any_rebuild = b->any_rebuild || k.rebuild;
    b->status_ptrs.back() = ib->d_status;
  }
  int rc;
  for (int c = 0; c < b->nc; ++c) {
    if (kin[c].empty()) continue;
    double *dk = nullptr;
    if ((rc = bupload(b, &dk, kin[c]))) { ib_batch_destroy(b); return rc; }
    hc[c].kin = dk;
  }
  double *rec = nullptr;
  if ((rc = bmalloc(b, &rec, (size_t)b->nc * b->rec_slots * 8)) || (rc = bmalloc(b, &b->d_steps, b->nc)) ||
      (rc = bmalloc(b, &b->d_tpart, 3 * std::max<size_t>(1, btiles.size())))) {
    ib_batch_destroy(b);
    return rc;
  }
  cudaMemsetAsync(rec, 0, (size_t)b->nc * b->rec_slots * 8 * sizeof(double), ctx->stream);
  cudaMemsetAsync(b->d_steps, 0, b->nc * sizeof(int), ctx->stream);
  {
    std::vector<int> lim(b->nc);
    for (int c = 0; c < b->nc; ++c) lim[c] = std::max(0, cases[c].limit);
    if ((rc = bupload(b, &b->d_limit, lim))) {
      ib_batch_destroy(b);
      return rc;
    }
  }
  b->d_rec = rec;
  for (int c = 0; c < b->nc; ++c) hc[c].rec = rec + (size_t)c * b->rec_slots * 8;
  b->total_m = moff.back();
  b->total_b = boff.back();
  {
    double *tw = nullptr;
    int4 *tc = nullptr;
    if ((rc = bmalloc(b, &tw, (size_t)std::max<int64_t>(1, b->total_m) * kTabStride)) ||
        (rc = bmalloc(b, &tc, (size_t)std::max<int64_t>(1, b->total_m)))) {
      ib_batch_destroy(b);
      return rc;
    }
    for (int c = 0; c < b->nc; ++c) {
      hc[c].tw = tw + (size_t)moff[c] * kTabStride;
      hc[c].tc = tc + moff[c];
    }
  }
  b->total_drows = (int64_t)dlist.size();
  b->total_rm = (int64_t)rlist.size();
  b->nbt = (int)btiles.size();
  b->ncg = (int)cgcase.size();
  if ((rc = bupload(b, &b->d_cases, hc)) || (rc = bupload(b, &b->d_bands, hb)) ||
      (rc = bupload(b, &b->d_mlist, mlist)) || (rc = bupload(b, &b->d_rlist, rlist)) ||
      (rc = bupload(b, &b->d_dlist, dlist)) || (rc = bupload(b, &b->d_btiles, btiles)) ||
      (rc = bupload(b, &b->d_cgcase, cgcase))) {
    ib_batch_destroy(b);
    return rc;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    ib_batch_destroy(b);
    return cuda_fail(e, "ib_batch_create");
  }
  *out = b;
  return ILBM_OK;
}

int ib_batch_forcing(IBBatch *b, const StepArgs *d_args, cudaStream_t s) {
  ilbm_ctx *ctx = b->ctx;
  if (b->total_m == 0) return ILBM_OK;
  const int *st = b->d_steps, *lm = b->d_limit;
  int rc = batch_band_macro_launch(ctx, d_args, b->d_bands, b->d_btiles, b->nbt, st, lm, s);
  if (rc) return rc;
  const int gt = std::min(b->nbt, 4096), gm = grid_for(b->total_m, 256);
  const int gw = grid_for(b->total_m * 32, 128), gr = grid_for(b->total_rm * 32, 128);
  const ItemRef *ml = b->d_mlist, *rl = b->d_rlist;
  const int64_t nm = b->total_m, nr = b->total_rm;
  // (the band macro also zeroed EFI)
  k_b_markers<<<gm, 256, 0, s>>>(b->d_cases, ml, nm, st, lm);
  ctx->launches += 1;
  if (b->any_periodic) {
    k_b_band<<<gt, kItemTile, 0, s>>>(b->d_cases, b->d_btiles, b->nbt, 1, st, lm);
    ctx->launches++;
  }
  k_b_marker_warp<0><<<gw, 128, 0, s>>>(b->d_cases, ml, nm, st, lm);
  ctx->launches++;
  // the moving bodies' operator build and CG (the longer chain) on the
  // high-priority side stream, the stored-inverse solves beside them
  const bool fork = b->ncg > 0 && b->total_drows > 0;
  cudaStream_t cgs = fork ? ctx->side : s;
  if (fork) {
    cudaError_t e = cudaEventRecord(b->ev_fork, s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(cgs, b->ev_fork, 0);
    if (e != cudaSuccess) return cuda_fail(e, "batched IVC fork");
  }
  if (nr > 0) {
    k_b_marker_warp<3><<<gr, 128, 0, cgs>>>(b->d_cases, rl, nr, st, lm);
    k_b_scan<<<b->ncg, kCgThreads, 0, cgs>>>(b->d_cases, b->d_cgcase, st, lm);
    k_b_marker_warp<4><<<gr, 128, 0, cgs>>>(b->d_cases, rl, nr, st, lm);
    ctx->launches += 3;
  }
  if (b->ncg > 0) {
    k_b_cg<<<b->ncg, kCgThreads, 0, cgs>>>(b->d_cases, b->d_cgcase, st, lm);
    ctx->launches++;
  }
  if (b->total_drows > 0) {
    k_b_dense<<<(unsigned)b->total_drows, kDenseThreads, 0, s>>>(b->d_cases, b->d_dlist, st, lm);
    ctx->launches++;
  }
  if (fork) {
    cudaError_t e = cudaEventRecord(b->ev_join, cgs);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, b->ev_join, 0);
    if (e != cudaSuccess) return cuda_fail(e, "batched IVC join");
  }
  if (b->any_explicit) {
    k_b_marker_warp<1><<<gw, 128, 0, s>>>(b->d_cases, ml, nm, st, lm);
    ctx->launches++;
  }
  k_b_marker_warp<2><<<gw, 128, 0, s>>>(b->d_cases, ml, nm, st, lm);
  ctx->launches++;
  if (b->any_periodic) {
    k_b_band<<<gt, kItemTile, 0, s>>>(b->d_cases, b->d_btiles, b->nbt, 2, st, lm);
    ctx->launches++;
  }
  if (ctx->storage == ILBM_STORAGE_F64)
    k_b_export<double><<<gt, kItemTile, 0, s>>>(b->d_cases, b->d_btiles, b->nbt, d_args, st, lm,
                                                 b->d_tpart);
  else
    k_b_export<float><<<gt, kItemTile, 0, s>>>(b->d_cases, b->d_btiles, b->nbt, d_args, st, lm,
                                                b->d_tpart);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "batched update_forcing");
  return ILBM_OK;
}

int ib_batch_record(IBBatch *b, const StepArgs *, cudaStream_t s) {
  if (b->nc == 0) return ILBM_OK;
  k_b_record<<<(unsigned)b->nc, kRecThreads, 0, s>>>(b->d_cases, b->d_steps, b->d_limit, b->rec_slots,
                                                    b->d_tpart);
  b->ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "batched force record");
  return ILBM_OK;
}

int ib_batch_read(IBBatch *b, std::vector<double> &rec, std::vector<int> &steps,
                  std::vector<int> &status, cudaStream_t s) {
  rec.assign((size_t)b->nc * b->rec_slots * 8, 0.0);
  steps.assign(b->nc, 0);
  status.assign(b->nc, 0);
  cudaMemcpyAsync(rec.data(), b->d_rec, rec.size() * sizeof(double), cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(steps.data(), b->d_steps, steps.size() * sizeof(int), cudaMemcpyDeviceToHost, s);
  for (int c = 0; c < b->nc; ++c)
    if (b->status_ptrs[c])
      cudaMemcpyAsync(&status[c], b->status_ptrs[c], sizeof(int), cudaMemcpyDeviceToHost, s);
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "batch record read-back");
  return ILBM_OK;
}

int ib_batch_rec_slots(const IBBatch *b) { return b->rec_slots; }
const int *ib_batch_steps(const IBBatch *b) { return b->d_steps; }
const int *ib_batch_limits(const IBBatch *b) { return b->d_limit; }

}  // namespace ilbm
