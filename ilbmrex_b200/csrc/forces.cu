// Force evaluation on the device: the Eulerian forcing integral of
// AmrCoreLBM::ComputeIBForce (Source/Core/AmrCoreLBM.cpp:489-509) and the
// link-wise momentum exchange of IBForceEval
// (Source/IBM/IBForceEval.cpp:28-191).  Both are two-stage reductions with a
// fixed summation order, so repeated calls return identical bits.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <vector>

#include "batch_internal.h"
#include "ilbm_common.cuh"

using namespace ilbm;

namespace {

constexpr int kRedBlocks = 296;  // 2 x 148 SMs
constexpr int kRedThreads = 256;

struct RegionArgs {
  int lo[3], n[3];
  int mgl[3];
  int64_t ms0, ms1, ms2;
  int dim;
};

template <class R>
__global__ void __launch_bounds__(kRedThreads) k_force_partial(RegionArgs a, const R *F,
                                                               double *partial) {
  __shared__ double sh[3][kRedThreads / 32];
  const int64_t total = (int64_t)a.n[0] * a.n[1] * a.n[2];
  const int64_t per = (total + gridDim.x - 1) / gridDim.x;
  const int64_t t0 = (int64_t)blockIdx.x * per, t1 = min(total, t0 + per);
  double acc[3] = {0.0, 0.0, 0.0};
  for (int64_t t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
    const int i = a.lo[0] + (int)(t % a.n[0]);
    const int j = a.lo[1] + (int)((t / a.n[0]) % a.n[1]);
    const int k = a.lo[2] + (int)(t / ((int64_t)a.n[0] * a.n[1]));
    const int64_t m = (int64_t)(i - a.mgl[0]) + (int64_t)(j - a.mgl[1]) * a.ms0 +
                      (int64_t)(k - a.mgl[2]) * a.ms1;
    acc[0] += double(F[m]);
    acc[1] += double(F[m + a.ms2]);
    if (a.dim == 3) acc[2] += double(F[m + 2 * a.ms2]);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int c = 0; c < 3; ++c) {
    double v = acc[c];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[c][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double s = 0.0;
    for (int w = 0; w < kRedThreads / 32; ++w) s += sh[threadIdx.x][w];
    partial[blockIdx.x * 3 + threadIdx.x] = s;
  }
}

// The same partial sums over several boxes: the regions' cells are taken as
// one sequence (region by region, each in i-fastest order) cut into equal
// chunks, one per block, so the summation order depends on the box list only.
struct SumRegion {
  RegionArgs a;
  const void *F;
};

template <class R>
__global__ void __launch_bounds__(kRedThreads) k_force_partial_multi(const SumRegion *__restrict__ regs,
                                                                     int nregs, const int64_t *off,
                                                                     double *partial) {
  __shared__ double sh[3][kRedThreads / 32];
  const int64_t total = off[nregs];
  const int64_t per = (total + gridDim.x - 1) / gridDim.x;
  const int64_t t0 = (int64_t)blockIdx.x * per, t1 = min(total, t0 + per);
  double acc[3] = {0.0, 0.0, 0.0};
  for (int64_t t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
    int r = 0, hi = nregs - 1;
    while (r < hi) {
      const int mid = (r + hi + 1) >> 1;
      if (off[mid] <= t) r = mid;
      else hi = mid - 1;
    }
    const RegionArgs &a = regs[r].a;
    const R *F = static_cast<const R *>(regs[r].F);
    const int64_t u = t - off[r];
    const int i = a.lo[0] + (int)(u % a.n[0]);
    const int j = a.lo[1] + (int)((u / a.n[0]) % a.n[1]);
    const int k = a.lo[2] + (int)(u / ((int64_t)a.n[0] * a.n[1]));
    const int64_t m = (int64_t)(i - a.mgl[0]) + (int64_t)(j - a.mgl[1]) * a.ms0 +
                      (int64_t)(k - a.mgl[2]) * a.ms1;
    acc[0] += double(F[m]);
    acc[1] += double(F[m + a.ms2]);
    if (a.dim == 3) acc[2] += double(F[m + 2 * a.ms2]);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int c = 0; c < 3; ++c) {
    double v = acc[c];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[c][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double s = 0.0;
    for (int w = 0; w < kRedThreads / 32; ++w) s += sh[threadIdx.x][w];
    partial[blockIdx.x * 3 + threadIdx.x] = s;
  }
}

// one warp: the partials' fixed-order total (lane l sums partials l, l + 32,
// ..., whose loads are in flight together, then a fixed butterfly); with rec
// set, also one force record: the total (3), the body's last marker force sum
// (3) and its two status words as doubles
__global__ void k_final_sum(const double *partial, int nparts, double *out,
                            const double *fsum = nullptr, const int *status = nullptr,
                            double *rec = nullptr) {
  const int lane = threadIdx.x & 31;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int b = lane; b < nparts; b += 32) {
    s0 += partial[b * 3];
    s1 += partial[b * 3 + 1];
    s2 += partial[b * 3 + 2];
  }
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if (threadIdx.x != 0) return;
  out[0] = s0;
  out[1] = s1;
  out[2] = s2;
  if (rec) {
    rec[0] = s0;
    rec[1] = s1;
    rec[2] = s2;
    for (int c = 0; c < 3; ++c) rec[3 + c] = fsum[c];
    rec[6] = (double)status[0];
    rec[7] = (double)status[1];
    __threadfence_system();  // rec may be pinned host memory the host reads next
  }
}

struct MEArgs {
  int dlo[3], dhi[3];
  int periodic[3];
  double plo[3], dx[3];
  double x0, y0, z0, R;
  int one_sided;
  float f16_scale;
  int nbox;
};

// one box of the level: valid region, allocated lower corner and strides of f
struct MEBox {
  int lo[3], hi[3], fgl[3];
  int64_t fs0, fs1, fs2;
  const void *f;
};

__device__ __forceinline__ double sdist(const MEArgs &a, int D, double x, double y, double z) {
  const double dx = X::sub(x, a.x0), dy = X::sub(y, a.y0);
  double s = X::add(X::mul(dx, dx), X::mul(dy, dy));
  if (D == 3) {
    const double dz = X::sub(z, a.z0);
    s = X::add(s, X::mul(dz, dz));
  }
  return X::sub(__dsqrt_rn(s), a.R);
}

__device__ __forceinline__ bool box_holds(const MEBox &b, int D, int i, int j, int k, int grow) {
  return i >= b.lo[0] - grow && i <= b.hi[0] + grow && j >= b.lo[1] - grow && j <= b.hi[1] + grow &&
         (D == 2 || (k >= b.lo[2] - grow && k <= b.hi[2] + grow));
}

// Link-wise momentum exchange over the valid cells of every box, taken as one
// sequence cut into equal chunks (fixed summation order for a given box
// list).  The population of a solid neighbour comes from the box whose valid
// region holds it, else from this box's caller-filled ghost layer; a link
// whose neighbour neither reaches is left out.
template <class L, int S>
__global__ void __launch_bounds__(kRedThreads) k_me_partial(MEArgs a, const MEBox *__restrict__ boxes,
                                                            const int64_t *off, double *partial) {
  using T = typename Store<S>::T;
  __shared__ double sh[3][kRedThreads / 32];
  const int64_t total = off[a.nbox];
  const int64_t per = (total + gridDim.x - 1) / gridDim.x;
  const int64_t t0 = (int64_t)blockIdx.x * per, t1 = min(total, t0 + per);
  double acc[3] = {0.0, 0.0, 0.0};
  auto load = [&](const MEBox &b, int i, int j, int k, int q) -> double {
    const int64_t e = (int64_t)(i - b.fgl[0]) + (int64_t)(j - b.fgl[1]) * b.fs0 +
                      (int64_t)(k - b.fgl[2]) * b.fs1 + q * b.fs2;
    const float s = (S == ILBM_STORAGE_F16_SCALED) ? float(L::w(q)) / a.f16_scale : 1.0f;
    double v = double(Store<S>::load(static_cast<const T *>(b.f) + e, s));
    if (Store<S>::shifted) v += L::w(q);
    return v;
  };
  const int nn[3] = {a.dhi[0] - a.dlo[0] + 1, a.dhi[1] - a.dlo[1] + 1, a.dhi[2] - a.dlo[2] + 1};
  for (int64_t t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
    int bi = 0, hi = a.nbox - 1;
    while (bi < hi) {
      const int mid = (bi + hi + 1) >> 1;
      if (off[mid] <= t) bi = mid;
      else hi = mid - 1;
    }
    const MEBox &B = boxes[bi];
    const int nx = B.hi[0] - B.lo[0] + 1, ny = B.hi[1] - B.lo[1] + 1;
    const int64_t u = t - off[bi];
    const int i = B.lo[0] + (int)(u % nx);
    const int j = B.lo[1] + (int)((u / nx) % ny);
    const int k = (L::D == 3) ? B.lo[2] + (int)(u / ((int64_t)nx * ny)) : 0;
    const double xc = X::add(a.plo[0], X::mul(X::add(double(i), 0.5), a.dx[0]));
    const double yc = X::add(a.plo[1], X::mul(X::add(double(j), 0.5), a.dx[1]));
    const double zc = (L::D == 3) ? X::add(a.plo[2], X::mul(X::add(double(k), 0.5), a.dx[2])) : 0.0;
    if (!(sdist(a, L::D, xc, yc, zc) > 0.0)) continue;
#pragma unroll
    for (int q = 1; q < L::Q; ++q) {
      int c[3] = {i + L::cx(q), j + L::cy(q), k + L::cz(q)};
      bool skip = false;
#pragma unroll
      for (int d = 0; d < L::D; ++d) {
        if (c[d] < a.dlo[d] || c[d] > a.dhi[d]) {
          if (a.periodic[d]) c[d] = (c[d] < a.dlo[d]) ? c[d] + nn[d] : c[d] - nn[d];
          else skip = true;
        }
      }
      if (skip) continue;
      if (L::D != 3) c[2] = 0;
      const double xn = X::add(a.plo[0], X::mul(X::add(double(c[0]), 0.5), a.dx[0]));
      const double yn = X::add(a.plo[1], X::mul(X::add(double(c[1]), 0.5), a.dx[1]));
      const double zn = (L::D == 3) ? X::add(a.plo[2], X::mul(X::add(double(c[2]), 0.5), a.dx[2])) : 0.0;
      if (!(sdist(a, L::D, xn, yn, zn) <= 0.0)) continue;
      const double fo = load(B, i, j, k, q);
      double dm;
      if (a.one_sided) {
        dm = X::mul(2.0, fo);
      } else {
        int src = box_holds(B, L::D, c[0], c[1], c[2], 0) ? bi : -1;
        for (int b = 0; b < a.nbox && src < 0; ++b)
          if (box_holds(boxes[b], L::D, c[0], c[1], c[2], 0)) src = b;
        if (src < 0 && box_holds(B, L::D, c[0], c[1], c[2], B.lo[0] - B.fgl[0])) src = bi;
        if (src < 0) continue;
        dm = X::add(fo, load(boxes[src], c[0], c[1], c[2], opposite<L>(q)));
      }
      acc[0] += dm * double(L::cx(q));
      acc[1] += dm * double(L::cy(q));
      acc[2] += dm * double(L::cz(q));
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int c = 0; c < 3; ++c) {
    double v = acc[c];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[c][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double s = 0.0;
    for (int w = 0; w < kRedThreads / 32; ++w) s += sh[threadIdx.x][w];
    partial[blockIdx.x * 3 + threadIdx.x] = s;
  }
}

template <class L, int S>
int launch_me(ilbm_ctx *ctx, const MEArgs &a, const MEBox *boxes, const int64_t *off,
              double *partial) {
  k_me_partial<L, S><<<kRedBlocks, kRedThreads, 0, ctx->stream>>>(a, boxes, off, partial);
  ctx->launches++;
  return ILBM_OK;
}

}  // namespace

extern "C" {

int ilbm_force_integrals(ilbm_ctx *ctx, const ilbm_box *boxes, int nbox, const int lo[3],
                         const int hi[3], double out_sum[3]) {
  if (!ctx || !boxes || nbox < 1 || !out_sum) {
    set_error("ilbm_force_integrals: null argument");
    return ILBM_ERR_ARG;
  }
  double *d_sum = nullptr;
  int rc = force_sum_enqueue(ctx, boxes, nbox, lo, hi, &d_sum);
  if (rc) return rc;
  cudaMemcpyAsync(ctx->host_pinned, d_sum, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_force_integrals");
  for (int c = 0; c < 3; ++c) out_sum[c] = ctx->host_pinned[c];
  return ILBM_OK;
}

}  // extern "C"

namespace ilbm {

// valid cells of `box` inside [lo, hi] (NULL: the whole box)
static RegionArgs clip_region(const ilbm_ctx *ctx, const ilbm_box &box, const int lo[3],
                              const int hi[3]) {
  RegionArgs a;
  std::memset(&a, 0, sizeof(a));
  a.dim = ctx->dim;
  for (int d = 0; d < 3; ++d) {
    if (d >= ctx->dim) {
      a.lo[d] = 0;
      a.n[d] = 1;
      a.mgl[d] = 0;
      continue;
    }
    const int l = std::max(lo ? lo[d] : box.lo[d], box.lo[d]);
    const int h = std::min(hi ? hi[d] : box.hi[d], box.hi[d]);
    a.lo[d] = l;
    a.n[d] = std::max(0, h - l + 1);
    a.mgl[d] = box.lo[d] - box.ngrow_m;
  }
  a.ms0 = box.mstride[0];
  a.ms1 = box.mstride[1];
  a.ms2 = box.mstride[2];
  return a;
}

int force_sum_enqueue(ilbm_ctx *ctx, const ilbm_box *boxes, int nbox, const int lo[3],
                      const int hi[3], double **d_sum, const double *fsum, const int *status,
                      double *rec_dst) {
  std::vector<SumRegion> regs;
  std::vector<int64_t> off(1, 0);
  for (int b = 0; b < nbox; ++b) {
    if (!boxes[b].force) {
      set_error("ilbm_force_integrals: box->force (the array to integrate) is required");
      return ILBM_ERR_ARG;
    }
    const RegionArgs a = clip_region(ctx, boxes[b], lo, hi);
    const int64_t cells = (int64_t)a.n[0] * a.n[1] * a.n[2];
    if (cells == 0) continue;
    regs.push_back({a, boxes[b].force});
    off.push_back(off.back() + cells);
  }
  const int nregs = (int)regs.size();
  // partials, the result (+ a record slot after it), then the region table
  const size_t head = (size_t)kRedBlocks * 3 + 16;
  const size_t table = nregs > 1 ? nregs * sizeof(SumRegion) + (nregs + 1) * sizeof(int64_t) : 0;
  double *scr = static_cast<double *>(ilbm_ctx_scratch(ctx, head * sizeof(double) + table + 16));
  if (!scr) {
    set_error("ilbm_force_integrals: scratch allocation failed");
    return ILBM_ERR_NOMEM;
  }
  *d_sum = scr + kRedBlocks * 3;
  // the record: rec_dst, else after the sums' spare slots
  double *rec = fsum ? (rec_dst ? rec_dst : *d_sum + 8) : nullptr;
  if (nregs == 0) {
    if (rec) {
      k_final_sum<<<1, 32, 0, ctx->stream>>>(scr, 0, *d_sum, fsum, status, rec);
      ctx->launches++;
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_fail(e, "ilbm_force_integrals");
      return ILBM_OK;
    }
    cudaError_t e = cudaMemsetAsync(*d_sum, 0, 3 * sizeof(double), ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "ilbm_force_integrals");
    return ILBM_OK;
  }
  const bool f64 = ctx->storage == ILBM_STORAGE_F64;
  if (nregs == 1) {
    if (f64)
      k_force_partial<double><<<kRedBlocks, kRedThreads, 0, ctx->stream>>>(
          regs[0].a, static_cast<const double *>(regs[0].F), scr);
    else
      k_force_partial<float><<<kRedBlocks, kRedThreads, 0, ctx->stream>>>(
          regs[0].a, static_cast<const float *>(regs[0].F), scr);
  } else {
    SumRegion *d_regs = reinterpret_cast<SumRegion *>(scr + head);
    int64_t *d_off = reinterpret_cast<int64_t *>(d_regs + nregs);
    cudaError_t e = cudaMemcpyAsync(d_regs, regs.data(), nregs * sizeof(SumRegion),
                                    cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_off, off.data(), (nregs + 1) * sizeof(int64_t), cudaMemcpyHostToDevice,
                          ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "ilbm_force_integrals: region table");
    if (f64)
      k_force_partial_multi<double><<<kRedBlocks, kRedThreads, 0, ctx->stream>>>(d_regs, nregs, d_off, scr);
    else
      k_force_partial_multi<float><<<kRedBlocks, kRedThreads, 0, ctx->stream>>>(d_regs, nregs, d_off, scr);
  }
  k_final_sum<<<1, 32, 0, ctx->stream>>>(scr, kRedBlocks, *d_sum, fsum, status, rec);
  ctx->launches += 2;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_force_integrals");
  return ILBM_OK;
}

// one box's force record (the region sum, fsum[0..2], status[0..1]) into rec
// (device-accessible) on stream st, with the caller's scratch (at least
// force_record_scratch() doubles): the launches of force_sum_enqueue for one
// region, in the same fixed order
size_t force_record_scratch() { return (size_t)kRedBlocks * 3 + 16; }

int force_record_on(ilbm_ctx *ctx, const ilbm_box &box, const int lo[3], const int hi[3],
                    const double *fsum, const int *status, double *rec, double *scr,
                    cudaStream_t st) {
  if (!box.force) {
    set_error("force record: box->force (the array to integrate) is required");
    return ILBM_ERR_ARG;
  }
  const RegionArgs a = clip_region(ctx, box, lo, hi);
  const int64_t cells = (int64_t)a.n[0] * a.n[1] * a.n[2];
  double *sum = scr + kRedBlocks * 3;
  int nparts = 0;
  if (cells > 0) {
    if (ctx->storage == ILBM_STORAGE_F64)
      k_force_partial<double><<<kRedBlocks, kRedThreads, 0, st>>>(a, static_cast<const double *>(box.force), scr);
    else
      k_force_partial<float><<<kRedBlocks, kRedThreads, 0, st>>>(a, static_cast<const float *>(box.force), scr);
    ctx->launches++;
    nparts = kRedBlocks;
  }
  k_final_sum<<<1, 32, 0, st>>>(scr, nparts, sum, fsum, status, rec);
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "force record");
  return ILBM_OK;
}

}  // namespace ilbm

extern "C" {

int ilbm_momentum_exchange(ilbm_ctx *ctx, const ilbm_box *boxes, int nbox,
                           const ilbm_level_params *p, double x0, double y0, double z0, double R,
                           const double prob_lo[3], const double dx[3], int one_sided,
                           double out[3]) {
  if (!ctx || !boxes || nbox < 1 || !p || !out || !prob_lo || !dx) {
    set_error("ilbm_momentum_exchange: null argument");
    return ILBM_ERR_ARG;
  }
  MEArgs a;
  std::memset(&a, 0, sizeof(a));
  for (int d = 0; d < 3; ++d) {
    const bool use = d < ctx->dim;
    a.dlo[d] = use ? p->domain_lo[d] : 0;
    a.dhi[d] = use ? p->domain_hi[d] : 0;
    a.periodic[d] = use ? p->periodic[d] : 0;
    a.plo[d] = prob_lo[d];
    a.dx[d] = dx[d];
  }
  a.x0 = x0;
  a.y0 = y0;
  a.z0 = (ctx->dim == 3) ? z0 : 0.0;
  a.R = R;
  a.one_sided = one_sided;
  a.f16_scale = (p->f16_scale > 0) ? float(p->f16_scale) : 1024.0f;
  a.nbox = nbox;
  std::vector<MEBox> mb(nbox);
  std::vector<int64_t> off(nbox + 1, 0);
  for (int b = 0; b < nbox; ++b) {
    const ilbm_box &x = boxes[b];
    if (!x.f_in) {
      set_error("ilbm_momentum_exchange: box->f_in is required");
      return ILBM_ERR_ARG;
    }
    int64_t cells = 1;
    for (int d = 0; d < 3; ++d) {
      const bool use = d < ctx->dim;
      mb[b].lo[d] = use ? x.lo[d] : 0;
      mb[b].hi[d] = use ? x.hi[d] : 0;
      mb[b].fgl[d] = use ? x.lo[d] - x.ngrow_f : 0;
      cells *= (int64_t)(mb[b].hi[d] - mb[b].lo[d] + 1);
    }
    if (cells <= 0) {
      set_error("ilbm_momentum_exchange: empty box");
      return ILBM_ERR_ARG;
    }
    mb[b].fs0 = x.fstride[0];
    mb[b].fs1 = x.fstride[1];
    mb[b].fs2 = x.fstride[2];
    mb[b].f = x.f_in;
    off[b + 1] = off[b] + cells;
  }
  const size_t head = (size_t)kRedBlocks * 3 + 8;
  char *scr = static_cast<char *>(ilbm_ctx_scratch(
      ctx, head * sizeof(double) + nbox * sizeof(MEBox) + (nbox + 1) * sizeof(int64_t)));
  if (!scr) {
    set_error("ilbm_momentum_exchange: scratch allocation failed");
    return ILBM_ERR_NOMEM;
  }
  double *part = reinterpret_cast<double *>(scr);
  MEBox *d_boxes = reinterpret_cast<MEBox *>(scr + head * sizeof(double));
  int64_t *d_off = reinterpret_cast<int64_t *>(d_boxes + nbox);
  cudaError_t e = cudaMemcpyAsync(d_boxes, mb.data(), nbox * sizeof(MEBox), cudaMemcpyHostToDevice,
                                  ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_off, off.data(), (nbox + 1) * sizeof(int64_t), cudaMemcpyHostToDevice,
                        ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_momentum_exchange: box table");
  int rc;
  switch (ctx->q * 4 + ctx->storage) {
    case 9 * 4 + 0: rc = launch_me<Lat<9>, 0>(ctx, a, d_boxes, d_off, part); break;
    case 9 * 4 + 1: rc = launch_me<Lat<9>, 1>(ctx, a, d_boxes, d_off, part); break;
    case 9 * 4 + 2: rc = launch_me<Lat<9>, 2>(ctx, a, d_boxes, d_off, part); break;
    case 19 * 4 + 0: rc = launch_me<Lat<19>, 0>(ctx, a, d_boxes, d_off, part); break;
    case 19 * 4 + 1: rc = launch_me<Lat<19>, 1>(ctx, a, d_boxes, d_off, part); break;
    case 19 * 4 + 2: rc = launch_me<Lat<19>, 2>(ctx, a, d_boxes, d_off, part); break;
    case 27 * 4 + 0: rc = launch_me<Lat<27>, 0>(ctx, a, d_boxes, d_off, part); break;
    case 27 * 4 + 1: rc = launch_me<Lat<27>, 1>(ctx, a, d_boxes, d_off, part); break;
    case 27 * 4 + 2: rc = launch_me<Lat<27>, 2>(ctx, a, d_boxes, d_off, part); break;
    default: set_error("unsupported lattice/storage"); return ILBM_ERR_UNSUPPORTED;
  }
  if (rc) return rc;
  k_final_sum<<<1, 32, 0, ctx->stream>>>(part, kRedBlocks, part + kRedBlocks * 3);
  ctx->launches++;
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_momentum_exchange");
  cudaMemcpyAsync(ctx->host_pinned, part + kRedBlocks * 3, 3 * sizeof(double),
                  cudaMemcpyDeviceToHost, ctx->stream);
  e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_momentum_exchange");
  for (int c = 0; c < 3; ++c) out[c] = -ctx->host_pinned[c];
  return ILBM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Force integral that allocates nothing
// ---------------------------------------------------------------------------
// ilbm_force_integrals grows the context's scratch with cudaMalloc on first
// use.  Some hosts cannot allocate once they are running: AMReX's default
// arena reserves most of the device memory at start-up, so a later cudaMalloc
// by a library can fail; a serving loop that admits cases against a fixed
// memory budget must not grow behind its back; and cudaMalloc / cudaFree can
// synchronise the device, stalling work queued on other streams.  This
// variant keeps its partial sums in a fixed array in the library's own
// device image instead.
//
// The region is cut into ceil(cells / kNoAllocChunkCells) equal chunks, one
// partial triple per chunk, so the summation order depends on the region
// only.  The array holds kNoAllocChunks partials plus the 3-double result:
// regions up to kNoAllocChunks * kNoAllocChunkCells cells (8,388,608).  Nothing in it has to start at
// zero: every partial that k_final_sum reads is written by k_force_partial
// earlier in the same call, and the result slot is written by k_final_sum.

namespace {

constexpr int kNoAllocChunks = 2048;
constexpr int64_t kNoAllocChunkCells = 4096;
constexpr int kNoAllocMaxDevices = 64;

__device__ __align__(256) double g_noalloc_scratch[kNoAllocChunks * 3 + 3];

// Device address of g_noalloc_scratch, looked up once per device.  Two host
// threads that make their first call on a device at the same time may both
// look it up; they store the same address, and the atomics make the store
// and the later loads well defined.  The address belongs to the device's
// primary context: after cudaDeviceReset every context of this library on
// that device is gone anyway, and the cache must not be used again (the
// header says so).
std::atomic<double *> g_noalloc_ptr[kNoAllocMaxDevices] = {};

int noalloc_scratch(int device, double **out) {
  if (device < 0 || device >= kNoAllocMaxDevices) {
    set_error("ilbm_force_integrals_noalloc: device ordinal out of range");
    return ILBM_ERR_ARG;
  }
  double *cached = g_noalloc_ptr[device].load(std::memory_order_acquire);
  if (!cached) {
    int prev = 0;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return cuda_fail(e, "ilbm_force_integrals_noalloc: cudaGetDevice");
    if (prev != device && (e = cudaSetDevice(device)) != cudaSuccess)
      return cuda_fail(e, "ilbm_force_integrals_noalloc: cudaSetDevice");
    void *ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (prev != device) cudaSetDevice(prev);
    if (e != cudaSuccess || !ptr)
      return cuda_fail(e != cudaSuccess ? e : cudaErrorInvalidSymbol,
                       "ilbm_force_integrals_noalloc: cudaGetSymbolAddress");
    cached = static_cast<double *>(ptr);
    g_noalloc_ptr[device].store(cached, std::memory_order_release);
  }
  *out = cached;
  return ILBM_OK;
}

}  // namespace

extern "C" {

int ilbm_force_integrals_noalloc(ilbm_ctx *ctx, const ilbm_box *box, const void *force,
                                 const int lo[3], const int hi[3], double out_sum[3]) {
  if (!ctx || !box || !force || !out_sum) {
    set_error("ilbm_force_integrals_noalloc: null argument");
    return ILBM_ERR_ARG;
  }
  RegionArgs a;
  std::memset(&a, 0, sizeof(a));
  a.dim = ctx->dim;
  for (int d = 0; d < 3; ++d) {
    if (d >= ctx->dim) {
      a.lo[d] = 0;
      a.n[d] = 1;
      a.mgl[d] = 0;
      continue;
    }
    const int l = std::max(lo ? lo[d] : box->lo[d], box->lo[d]);
    const int h = std::min(hi ? hi[d] : box->hi[d], box->hi[d]);
    a.lo[d] = l;
    a.n[d] = std::max(0, h - l + 1);
    a.mgl[d] = box->lo[d] - box->ngrow_m;
  }
  a.ms0 = box->mstride[0];
  a.ms1 = box->mstride[1];
  a.ms2 = box->mstride[2];
  const int64_t cells = (int64_t)a.n[0] * a.n[1] * a.n[2];
  const int64_t max_cells = (int64_t)kNoAllocChunks * kNoAllocChunkCells;
  if (cells > max_cells) {
    char msg[200];
    std::snprintf(msg, sizeof(msg),
                  "ilbm_force_integrals_noalloc: region has %lld cells; the static scratch covers at "
                  "most %lld (%d chunks of %lld cells); use ilbm_force_integrals",
                  (long long)cells, (long long)max_cells, kNoAllocChunks,
                  (long long)kNoAllocChunkCells);
    set_error(msg);
    return ILBM_ERR_RANGE;
  }
  double *scr = nullptr;
  int rc = noalloc_scratch(ctx->device, &scr);
  if (rc) return rc;
  if (cells == 0) {
    out_sum[0] = out_sum[1] = out_sum[2] = 0.0;
    return ILBM_OK;
  }
  const int nchunks = (int)((cells + kNoAllocChunkCells - 1) / kNoAllocChunkCells);
  if (ctx->storage == ILBM_STORAGE_F64)
    k_force_partial<double><<<nchunks, kRedThreads, 0, ctx->stream>>>(a, static_cast<const double *>(force), scr);
  else
    k_force_partial<float><<<nchunks, kRedThreads, 0, ctx->stream>>>(a, static_cast<const float *>(force), scr);
  k_final_sum<<<1, 32, 0, ctx->stream>>>(scr, nchunks, scr + kNoAllocChunks * 3);
  ctx->launches += 2;
  // a launch that failed without poisoning the context (bad configuration,
  // missing kernel image) is not reported by the synchronisation below; the
  // result slot would then still hold the previous call's sum
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_force_integrals_noalloc: launch");
  double res[3] = {0.0, 0.0, 0.0};
  e = cudaMemcpyAsync(res, scr + kNoAllocChunks * 3, 3 * sizeof(double), cudaMemcpyDeviceToHost,
                      ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_force_integrals_noalloc: copy");
  e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_force_integrals_noalloc");
  for (int c = 0; c < 3; ++c) out_sum[c] = res[c];
  return ILBM_OK;
}

}  // extern "C"
