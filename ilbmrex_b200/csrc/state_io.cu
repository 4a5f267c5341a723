// State I/O of one level box: checkpoint / restart (with the immersed body)
// and the AMReX plotfile writer.
//
// Device side: gathers of the valid cells of a ghosted Array4-layout array
// into dense component planes (i fastest) and the scatter back, and the
// plotfile's component planes in FP64 (macro fields, vorticity, pressure,
// unshifted populations, the body's level set).  Host side: one component
// plane at a time through two device and two pinned host buffers, so the
// file write of plane c overlaps the gather and copy of plane c + 1.

#include <sys/stat.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ilbm_common.cuh"
#include "state_internal.h"

namespace ilbm {
namespace {

// valid cells of one box inside a ghosted array
struct Plane {
  int nx, ny, nz;
  int64_t s0, s1;  // j and k strides (elements)
  int64_t origin;  // element offset of the box's lo cell from the array start
  __host__ __device__ int64_t cells() const { return (int64_t)nx * ny * nz; }
};

Plane plane_of(const ilbm_box *box, int dim, int ngrow, const int64_t *stride) {
  Plane p;
  p.nx = box->hi[0] - box->lo[0] + 1;
  p.ny = box->hi[1] - box->lo[1] + 1;
  p.nz = (dim == 3) ? box->hi[2] - box->lo[2] + 1 : 1;
  p.s0 = stride[0];
  p.s1 = stride[1];
  p.origin = ngrow + (int64_t)ngrow * stride[0] + ((dim == 3) ? (int64_t)ngrow * stride[1] : 0);
  return p;
}

__device__ __forceinline__ int64_t plane_off(const Plane &p, int64_t t, int &i, int &j, int &k) {
  i = (int)(t % p.nx);
  const int64_t r = t / p.nx;
  j = (int)(r % p.ny);
  k = (int)(r / p.ny);
  return p.origin + i + (int64_t)j * p.s0 + (int64_t)k * p.s1;
}

template <class T>
__global__ void __launch_bounds__(256) k_gather_plane(Plane p, const T *__restrict__ src,
                                                      T *__restrict__ dst) {
  const int64_t n = p.cells();
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    int i, j, k;
    dst[t] = src[plane_off(p, t, i, j, k)];
  }
}

template <class T>
__global__ void __launch_bounds__(256) k_scatter_plane(Plane p, const T *__restrict__ src,
                                                       T *__restrict__ dst) {
  const int64_t n = p.cells();
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    int i, j, k;
    dst[plane_off(p, t, i, j, k)] = src[t];
  }
}

struct PlotArgs {
  Plane pl;
  int dim;
  int lo[3];
  double plo[3], dx[3];
  int mask;
  double c[3], R;
  double ub[3];
};

// signed distance of the cell centre to the body (LevelSetManager::
// build_from_cylinder, Source/LevelSet/LevelSet.cpp:56-70)
__device__ __forceinline__ double phi_at(const PlotArgs &a, int i, int j, int k) {
  const double x = X::add(a.plo[0], X::mul(X::add(double(a.lo[0] + i), 0.5), a.dx[0]));
  const double y = X::add(a.plo[1], X::mul(X::add(double(a.lo[1] + j), 0.5), a.dx[1]));
  const double ex = X::sub(x, a.c[0]), ey = X::sub(y, a.c[1]);
  double r2 = X::add(X::mul(ex, ex), X::mul(ey, ey));
  if (a.dim == 3) {
    const double z = X::add(a.plo[2], X::mul(X::add(double(a.lo[2] + k), 0.5), a.dx[2]));
    const double ez = X::sub(z, a.c[2]);
    r2 = X::add(r2, X::mul(ez, ez));
  }
  return X::sub(__dsqrt_rn(r2), a.R);
}

// a real-typed macro-layout plane (NULL: zeros); kind 0: rho / Pressure,
// 1..3: ux, uy, uz (masked to the body velocity), 4: vorticity (masked to 0)
template <class R>
__global__ void __launch_bounds__(256) k_plot_real(PlotArgs a, const R *__restrict__ src, int kind,
                                                   double *__restrict__ dst) {
  const int64_t n = a.pl.cells();
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    int i, j, k;
    const int64_t m = plane_off(a.pl, t, i, j, k);
    double v = src ? double(src[m]) : 0.0;
    if (a.mask && kind >= 1 && kind <= 4 && phi_at(a, i, j, k) < 0.0)
      v = (kind <= 3) ? a.ub[kind - 1] : 0.0;
    dst[t] = v;
  }
}

// population q in its unshifted FP64 value: f, g + w, or h * (w / scale) + w
template <int S>
__global__ void __launch_bounds__(256) k_plot_pop(Plane pl, const typename Store<S>::T *__restrict__ f,
                                                  double w, double s, double *__restrict__ dst) {
  const int64_t n = pl.cells();
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    int i, j, k;
    const auto v = f[plane_off(pl, t, i, j, k)];
    double d;
    if (S == ILBM_STORAGE_F64)
      d = double(v);
    else if (S == ILBM_STORAGE_F32_SHIFT)
      d = X::add(double(v), w);
    else
      d = X::add(X::mul(double(__half2float(v)), s), w);
    dst[t] = d;
  }
}

__global__ void __launch_bounds__(256) k_plot_phi(PlotArgs a, double *__restrict__ dst) {
  const int64_t n = a.pl.cells();
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (int64_t)gridDim.x * blockDim.x) {
    int i, j, k;
    plane_off(a.pl, t, i, j, k);
    dst[t] = phi_at(a, i, j, k);
  }
}

int grid_for(const ilbm_ctx *ctx, int64_t n) {
  const int64_t cap = (int64_t)std::max(ctx->sms, 1) * 16;
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, cap));
}

// 64-bit word hash of a byte stream fed in pieces (multiply-xorshift per
// 8-byte word, the length folded in at the end)
struct Hasher {
  uint64_t h = 0x243F6A8885A308D3ull;
  uint64_t total = 0;
  unsigned char tail[8];
  int nt = 0;
  void word(uint64_t w) {
    h = (h ^ w) * 0x9E3779B97F4A7C15ull;
    h ^= h >> 32;
  }
  void add(const void *p, size_t n) {
    const unsigned char *b = static_cast<const unsigned char *>(p);
    total += n;
    while (n && nt) {
      tail[nt++] = *b++;
      --n;
      if (nt == 8) {
        uint64_t w;
        std::memcpy(&w, tail, 8);
        word(w);
        nt = 0;
      }
    }
    for (; n >= 8; n -= 8, b += 8) {
      uint64_t w;
      std::memcpy(&w, b, 8);
      word(w);
    }
    while (n--) tail[nt++] = *b++;
  }
  uint64_t done() {
    if (nt) {
      std::memset(tail + nt, 0, 8 - nt);
      uint64_t w;
      std::memcpy(&w, tail, 8);
      word(w);
      nt = 0;
    }
    word(total);
    return h;
  }
};

// two device planes and two pinned host planes with their events
struct Stage {
  void *d[2] = {nullptr, nullptr};
  void *h[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  size_t bytes = 0;
  ~Stage() {
    for (int s = 0; s < 2; ++s) {
      if (ev[s]) cudaEventDestroy(ev[s]);
      if (d[s]) cudaFree(d[s]);
      if (h[s]) cudaFreeHost(h[s]);
    }
  }
  int init(size_t n) {
    bytes = std::max<size_t>(n, 16);
    for (int s = 0; s < 2; ++s) {
      cudaError_t e = cudaMalloc(&d[s], bytes);
      if (e == cudaSuccess) e = cudaHostAlloc(&h[s], bytes, cudaHostAllocDefault);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev[s], cudaEventDisableTiming);
      if (e != cudaSuccess) return cuda_fail(e, "state I/O staging buffers");
    }
    return ILBM_OK;
  }
};

int io_fail(const std::string &what) {
  set_error(what + (errno ? std::string(": ") + std::strerror(errno) : std::string()));
  return ILBM_ERR_IO;
}

// ---- checkpoint file layout ----------------------------------------------
constexpr char kMagic[8] = {'I', 'L', 'B', 'M', 'C', 'K', 'P', 'T'};
constexpr uint32_t kVersion = 1;

struct CkptHeader {
  char magic[8];
  uint32_t version;
  uint32_t header_bytes;
  int32_t dim, q, storage, nsec;
  int32_t lo[3], hi[3];
  int64_t n_markers;
  int32_t cg_warm, flags;
  int64_t istep;
  double time;
  double user[16];
};

struct SecHeader {
  char tag[4];
  uint32_t elem_bytes;
  uint64_t ncomp;
  uint64_t count;  // elements per component
};

bool tag_is(const SecHeader &s, const char *t) { return std::memcmp(s.tag, t, 4) == 0; }

template <class T>
void launch_gather(ilbm_ctx *ctx, const Plane &pl, const void *src, void *dst) {
  k_gather_plane<T><<<grid_for(ctx, pl.cells()), 256, 0, ctx->stream>>>(
      pl, static_cast<const T *>(src), static_cast<T *>(dst));
  ctx->launches++;
}
template <class T>
void launch_scatter(ilbm_ctx *ctx, const Plane &pl, const void *src, void *dst) {
  k_scatter_plane<T><<<grid_for(ctx, pl.cells()), 256, 0, ctx->stream>>>(
      pl, static_cast<const T *>(src), static_cast<T *>(dst));
  ctx->launches++;
}

void gather_any(ilbm_ctx *ctx, int eb, const Plane &pl, const void *src, void *dst) {
  if (eb == 8) launch_gather<uint64_t>(ctx, pl, src, dst);
  else if (eb == 4) launch_gather<uint32_t>(ctx, pl, src, dst);
  else launch_gather<uint16_t>(ctx, pl, src, dst);
}
void scatter_any(ilbm_ctx *ctx, int eb, const Plane &pl, const void *src, void *dst) {
  if (eb == 8) launch_scatter<uint64_t>(ctx, pl, src, dst);
  else if (eb == 4) launch_scatter<uint32_t>(ctx, pl, src, dst);
  else launch_scatter<uint16_t>(ctx, pl, src, dst);
}

// ncomp component planes of a ghosted array (component stride cs elements)
int write_planes(ilbm_ctx *ctx, FILE *fp, const char *tag, const void *base, int64_t cs,
                 const Plane &pl, int ncomp, int eb, Stage &st) {
  SecHeader sh;
  std::memcpy(sh.tag, tag, 4);
  sh.elem_bytes = (uint32_t)eb;
  sh.ncomp = (uint64_t)ncomp;
  sh.count = (uint64_t)pl.cells();
  if (std::fwrite(&sh, sizeof(sh), 1, fp) != 1) return io_fail("checkpoint write");
  const size_t nb = (size_t)pl.cells() * eb;
  Hasher hs;
  const char *b = static_cast<const char *>(base);
  for (int c = 0; c <= ncomp; ++c) {
    if (c < ncomp) {
      const int s = c & 1;
      gather_any(ctx, eb, pl, b + (size_t)c * cs * eb, st.d[s]);
      cudaMemcpyAsync(st.h[s], st.d[s], nb, cudaMemcpyDeviceToHost, ctx->stream);
      cudaEventRecord(st.ev[s], ctx->stream);
    }
    if (c > 0) {
      const int s = (c - 1) & 1;
      cudaError_t e = cudaEventSynchronize(st.ev[s]);
      if (e != cudaSuccess) return cuda_fail(e, "checkpoint gather");
      hs.add(st.h[s], nb);
      if (std::fwrite(st.h[s], 1, nb, fp) != nb) return io_fail("checkpoint write");
    }
  }
  const uint64_t h = hs.done();
  if (std::fwrite(&h, sizeof(h), 1, fp) != 1) return io_fail("checkpoint write");
  return ILBM_OK;
}

int write_small(ilbm_ctx *ctx, FILE *fp, const char *tag, const double *dev, size_t n) {
  std::vector<double> h(std::max<size_t>(n, 1));
  cudaError_t e = cudaMemcpyAsync(h.data(), dev, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "checkpoint read-back of the body");
  SecHeader sh;
  std::memcpy(sh.tag, tag, 4);
  sh.elem_bytes = 8;
  sh.ncomp = 1;
  sh.count = n;
  Hasher hs;
  hs.add(h.data(), n * sizeof(double));
  const uint64_t hv = hs.done();
  if (std::fwrite(&sh, sizeof(sh), 1, fp) != 1 ||
      std::fwrite(h.data(), sizeof(double), n, fp) != n || std::fwrite(&hv, sizeof(hv), 1, fp) != 1)
    return io_fail("checkpoint write");
  return ILBM_OK;
}

int read_planes(ilbm_ctx *ctx, FILE *fp, const SecHeader &sh, void *base, int64_t cs,
                const Plane &pl, Stage &st) {
  const int eb = (int)sh.elem_bytes;
  const size_t nb = (size_t)pl.cells() * eb;
  Hasher hs;
  char *b = static_cast<char *>(base);
  for (int c = 0; c < (int)sh.ncomp; ++c) {
    const int s = c & 1;
    if (c >= 2) {
      cudaError_t e = cudaEventSynchronize(st.ev[s]);  // plane c - 2 has left this buffer
      if (e != cudaSuccess) return cuda_fail(e, "checkpoint scatter");
    }
    if (std::fread(st.h[s], 1, nb, fp) != nb) return io_fail("checkpoint read: short file");
    hs.add(st.h[s], nb);
    cudaMemcpyAsync(st.d[s], st.h[s], nb, cudaMemcpyHostToDevice, ctx->stream);
    scatter_any(ctx, eb, pl, st.d[s], b + (size_t)c * cs * eb);
    cudaEventRecord(st.ev[s], ctx->stream);
  }
  uint64_t h = 0;
  if (std::fread(&h, sizeof(h), 1, fp) != 1) return io_fail("checkpoint read: short file");
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "checkpoint scatter");
  if (h != hs.done()) {
    errno = 0;
    return io_fail(std::string("checkpoint read: hash mismatch in section ") +
                   std::string(sh.tag, 4));
  }
  return ILBM_OK;
}

int read_small(ilbm_ctx *ctx, FILE *fp, const SecHeader &sh, double *dev) {
  const size_t n = sh.count;
  std::vector<double> h(std::max<size_t>(n, 1));
  uint64_t hv = 0;
  if (std::fread(h.data(), sizeof(double), n, fp) != n || std::fread(&hv, sizeof(hv), 1, fp) != 1)
    return io_fail("checkpoint read: short file");
  Hasher hs;
  hs.add(h.data(), n * sizeof(double));
  if (hv != hs.done()) {
    errno = 0;
    return io_fail(std::string("checkpoint read: hash mismatch in section ") +
                   std::string(sh.tag, 4));
  }
  cudaError_t e = cudaMemcpyAsync(dev, h.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "checkpoint upload of the body");
  return ILBM_OK;
}

int real_bytes(const ilbm_ctx *ctx) { return ctx->storage == ILBM_STORAGE_F64 ? 8 : 4; }
int store_bytes(const ilbm_ctx *ctx) {
  return ctx->storage == ILBM_STORAGE_F64 ? 8 : (ctx->storage == ILBM_STORAGE_F32_SHIFT ? 4 : 2);
}

struct FileCloser {
  FILE *fp;
  ~FileCloser() {
    if (fp) std::fclose(fp);
  }
};

int check_box(const ilbm_ctx *ctx, const ilbm_box *box, const char *who) {
  for (int d = 0; d < ctx->dim; ++d)
    if (box->hi[d] < box->lo[d]) {
      set_error(std::string(who) + ": empty box");
      return ILBM_ERR_ARG;
    }
  if (box->fstride[0] <= 0 || box->fstride[1] <= 0 || box->fstride[2] <= 0) {
    set_error(std::string(who) + ": f strides must be positive");
    return ILBM_ERR_ARG;
  }
  if ((box->macro_in || box->force_prev) &&
      (box->mstride[0] <= 0 || box->mstride[1] <= 0 || box->mstride[2] <= 0)) {
    set_error(std::string(who) + ": macro strides must be positive");
    return ILBM_ERR_ARG;
  }
  return ILBM_OK;
}

// ---- plotfile text -------------------------------------------------------
std::string box_text(int dim, const int *lo, const int *hi) {
  char b[256];
  if (dim == 3)
    std::snprintf(b, sizeof(b), "((%d,%d,%d) (%d,%d,%d) (0,0,0))", lo[0], lo[1], lo[2], hi[0], hi[1],
                  hi[2]);
  else
    std::snprintf(b, sizeof(b), "((%d,%d) (%d,%d) (0,0))", lo[0], lo[1], hi[0], hi[1]);
  return b;
}

std::string num(double v) {
  char b[64];
  std::snprintf(b, sizeof(b), "%.17g", v);
  return b;
}

bool make_dir(const std::string &d) { return ::mkdir(d.c_str(), 0755) == 0 || errno == EEXIST; }

bool write_text(const std::string &path, const std::string &text) {
  FILE *fp = std::fopen(path.c_str(), "wb");
  if (!fp) return false;
  const bool ok = std::fwrite(text.data(), 1, text.size(), fp) == text.size();
  return (std::fclose(fp) == 0) && ok;
}

}  // namespace
}  // namespace ilbm

using namespace ilbm;

extern "C" {

int ilbm_checkpoint_write(ilbm_ctx *ctx, const ilbm_box *box, ilbm_ib *ib,
                          const ilbm_checkpoint_meta *meta, const char *path) {
  if (!ctx || !box || !box->f_in || !meta || !path) {
    set_error("ilbm_checkpoint_write: null argument");
    return ILBM_ERR_ARG;
  }
  int rc = check_box(ctx, box, "ilbm_checkpoint_write");
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  const Plane pf = plane_of(box, ctx->dim, box->ngrow_f, box->fstride);
  const Plane pm = plane_of(box, ctx->dim, box->ngrow_m, box->mstride);
  IBState bs;
  if (ib) ib_state(ib, &bs);
  CkptHeader hd;
  std::memset(&hd, 0, sizeof(hd));
  std::memcpy(hd.magic, kMagic, 8);
  hd.version = kVersion;
  hd.header_bytes = sizeof(CkptHeader);
  hd.dim = ctx->dim;
  hd.q = ctx->q;
  hd.storage = ctx->storage;
  for (int d = 0; d < 3; ++d) {
    hd.lo[d] = d < ctx->dim ? box->lo[d] : 0;
    hd.hi[d] = d < ctx->dim ? box->hi[d] : 0;
  }
  hd.flags = (box->macro_in ? ILBM_CKPT_MACRO : 0) | (box->force_prev ? ILBM_CKPT_FORCE : 0) |
             (ib ? ILBM_CKPT_BODY : 0);
  hd.nsec = 1 + (box->macro_in ? 1 : 0) + (box->force_prev ? 1 : 0) +
            (ib ? 4 + (bs.X ? 1 : 0) + (bs.Xh ? 1 : 0) : 0);
  hd.n_markers = ib ? bs.n : 0;
  hd.cg_warm = (ib && bs.cg_warm) ? (bs.cg_hist2 ? 3 : 1) : 0;  // bit 1: CG history
  hd.istep = meta->istep;
  hd.time = meta->time;
  std::memcpy(hd.user, meta->user, sizeof(hd.user));
  Stage st;
  if ((rc = st.init((size_t)pf.cells() * 8))) return rc;
  // everything queued on the stream (the last step, the body's chain) first
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_checkpoint_write");
  const std::string tmp = std::string(path) + ".tmp";
  errno = 0;
  FILE *fp = std::fopen(tmp.c_str(), "wb");
  if (!fp) return io_fail("ilbm_checkpoint_write: cannot create " + tmp);
  {
    FileCloser fc{fp};
    if (std::fwrite(&hd, sizeof(hd), 1, fp) != 1) return io_fail("checkpoint write");
    if ((rc = write_planes(ctx, fp, "FPOP", box->f_in, box->fstride[2], pf, ctx->q, store_bytes(ctx), st)))
      return rc;
    if (box->macro_in &&
        (rc = write_planes(ctx, fp, "MACR", box->macro_in, box->mstride[2], pm, 4, real_bytes(ctx), st)))
      return rc;
    if (box->force_prev &&
        (rc = write_planes(ctx, fp, "FPRV", box->force_prev, box->mstride[2], pm, 3, real_bytes(ctx), st)))
      return rc;
    if (ib) {
      const size_t n3 = 3 * (size_t)bs.n;
      if ((rc = write_small(ctx, fp, "MXYZ", bs.xyz, n3)) || (rc = write_small(ctx, fp, "MUVW", bs.uvw, n3)) ||
          (rc = write_small(ctx, fp, "MFRC", bs.F, n3)) || (rc = write_small(ctx, fp, "MSUM", bs.fsum, 3)))
        return rc;
      if (bs.X && (rc = write_small(ctx, fp, "MCGX", bs.X, n3))) return rc;
      if (bs.Xh && (rc = write_small(ctx, fp, "MCGH", bs.Xh, n3))) return rc;
    }
    if (std::fflush(fp) != 0) return io_fail("checkpoint write");
    fc.fp = nullptr;
    if (std::fclose(fp) != 0) return io_fail("checkpoint write");
  }
  if (std::rename(tmp.c_str(), path) != 0) return io_fail(std::string("checkpoint rename to ") + path);
  return ILBM_OK;
}

int ilbm_checkpoint_read(ilbm_ctx *ctx, const ilbm_box *box, ilbm_ib *ib, ilbm_checkpoint_meta *meta,
                         const char *path) {
  if (!ctx || !box || !box->f_in || !meta || !path) {
    set_error("ilbm_checkpoint_read: null argument");
    return ILBM_ERR_ARG;
  }
  int rc = check_box(ctx, box, "ilbm_checkpoint_read");
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  errno = 0;
  FILE *fp = std::fopen(path, "rb");
  if (!fp) return io_fail(std::string("ilbm_checkpoint_read: cannot open ") + path);
  FileCloser fc{fp};
  CkptHeader hd;
  if (std::fread(&hd, sizeof(hd), 1, fp) != 1) return io_fail("checkpoint read: short file");
  if (std::memcmp(hd.magic, kMagic, 8) != 0 || hd.version != kVersion ||
      hd.header_bytes != sizeof(CkptHeader)) {
    errno = 0;
    return io_fail("checkpoint read: not a checkpoint of this library (magic / version)");
  }
  auto mismatch = [&](const std::string &what) {
    set_error("ilbm_checkpoint_read: " + what);
    return ILBM_ERR_ARG;
  };
  if (hd.dim != ctx->dim || hd.q != ctx->q || hd.storage != ctx->storage)
    return mismatch("lattice or storage differs from the context");
  for (int d = 0; d < ctx->dim; ++d)
    if (hd.lo[d] != box->lo[d] || hd.hi[d] != box->hi[d]) return mismatch("box differs");
  if ((hd.flags & ILBM_CKPT_MACRO) && !box->macro_in)
    return mismatch("the file holds stored macro fields; box->macro_in is NULL");
  if (((hd.flags & ILBM_CKPT_FORCE) != 0) != (box->force_prev != nullptr))
    return mismatch("F^{n-1} present in only one of the file and box->force_prev");
  IBState bs;
  if (((hd.flags & ILBM_CKPT_BODY) != 0) != (ib != nullptr))
    return mismatch("an immersed body present in only one of the file and the call");
  if (ib) {
    ib_state(ib, &bs);
    if (hd.n_markers != bs.n) return mismatch("the body's marker count differs");
  }
  const Plane pf = plane_of(box, ctx->dim, box->ngrow_f, box->fstride);
  const Plane pm = plane_of(box, ctx->dim, box->ngrow_m, box->mstride);
  Stage st;
  if ((rc = st.init((size_t)pf.cells() * 8))) return rc;
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_checkpoint_read");
  bool got_cgx = false, got_cgh = false;
  for (int s = 0; s < hd.nsec; ++s) {
    SecHeader sh;
    if (std::fread(&sh, sizeof(sh), 1, fp) != 1) return io_fail("checkpoint read: short file");
    auto want = [&](uint64_t ncomp, uint64_t count, int eb) {
      return sh.ncomp == ncomp && sh.count == count && (int)sh.elem_bytes == eb;
    };
    if (tag_is(sh, "FPOP")) {
      if (!want(ctx->q, pf.cells(), store_bytes(ctx))) return mismatch("population section shape");
      if ((rc = read_planes(ctx, fp, sh, box->f_in, box->fstride[2], pf, st))) return rc;
    } else if (tag_is(sh, "MACR")) {
      if (!want(4, pm.cells(), real_bytes(ctx))) return mismatch("macro section shape");
      if ((rc = read_planes(ctx, fp, sh, box->macro_in, box->mstride[2], pm, st))) return rc;
    } else if (tag_is(sh, "FPRV")) {
      if (!want(3, pm.cells(), real_bytes(ctx))) return mismatch("force section shape");
      if ((rc = read_planes(ctx, fp, sh, box->force_prev, box->mstride[2], pm, st))) return rc;
    } else if (ib && (tag_is(sh, "MXYZ") || tag_is(sh, "MUVW") || tag_is(sh, "MFRC") ||
                      tag_is(sh, "MSUM") || tag_is(sh, "MCGX") || tag_is(sh, "MCGH"))) {
      const bool sum = tag_is(sh, "MSUM");
      if (!want(1, sum ? 3 : 3 * (uint64_t)bs.n, 8)) return mismatch("body section shape");
      double *dst = tag_is(sh, "MXYZ") ? bs.xyz
                    : tag_is(sh, "MUVW") ? bs.uvw
                    : tag_is(sh, "MFRC") ? bs.F
                    : sum                ? bs.fsum
                    : tag_is(sh, "MCGX") ? bs.X
                                         : bs.Xh;
      if (!dst) return mismatch("the file holds a CG start vector this body does not use");
      if ((rc = read_small(ctx, fp, sh, dst))) return rc;
      got_cgx = got_cgx || tag_is(sh, "MCGX");
      got_cgh = got_cgh || tag_is(sh, "MCGH");
    } else {
      return mismatch(std::string("unknown section ") + std::string(sh.tag, 4));
    }
  }
  if (ib) ib_set_cg_warm(ib, (hd.cg_warm & 1) && got_cgx, (hd.cg_warm & 2) && got_cgh);
  meta->istep = hd.istep;
  meta->time = hd.time;
  meta->flags = hd.flags;
  std::memcpy(meta->user, hd.user, sizeof(hd.user));
  return ILBM_OK;
}

int ilbm_plotfile_write(ilbm_ctx *ctx, const ilbm_box *box, const ilbm_level_params *p,
                        const ilbm_plot_info *info, const char *dir) {
  if (!ctx || !box || !box->f_in || !p || !info || !dir) {
    set_error("ilbm_plotfile_write: null argument");
    return ILBM_ERR_ARG;
  }
  int rc = check_box(ctx, box, "ilbm_plotfile_write");
  if (rc) return rc;
  if (box->mstride[0] <= 0 || box->mstride[1] <= 0 || box->mstride[2] <= 0) {
    set_error("ilbm_plotfile_write: macro strides (of the scratch planes) must be positive");
    return ILBM_ERR_ARG;
  }
  cudaSetDevice(ctx->device);
  const int dim = ctx->dim, Q = ctx->q;
  const Plane pf = plane_of(box, dim, box->ngrow_f, box->fstride);
  const Plane pm = plane_of(box, dim, box->ngrow_m, box->mstride);
  const int64_t N = pf.cells();
  const int rb = real_bytes(ctx);
  const int ncomp = 6 + Q + (info->levelset ? 1 : 0);
  // rho,u,v,w then vor, Pressure in the macro layout of the box
  const int64_t cs = box->mstride[2];
  void *mac = nullptr;
  cudaError_t e = cudaMalloc(&mac, (size_t)6 * cs * rb);
  if (e != cudaSuccess) return cuda_fail(e, "ilbm_plotfile_write scratch");
  struct Free {
    void *q;
    ~Free() { cudaFree(q); }
  } fr{mac};
  char *mb = static_cast<char *>(mac);
  if ((rc = ilbm_compute_macro(ctx, box, p, box->f_in, box->force_prev, mac, nullptr, nullptr)))
    return rc;
  double vmax = 0.0;
  if ((rc = ilbm_derived_fields(ctx, box, p, box->f_in, box->force_prev, info->dx, mb + 4 * cs * rb,
                                mb + 5 * cs * rb, &vmax)))
    return rc;
  PlotArgs a;
  std::memset(&a, 0, sizeof(a));
  a.pl = pm;
  a.dim = dim;
  for (int d = 0; d < 3; ++d) {
    a.lo[d] = d < dim ? box->lo[d] : 0;
    a.plo[d] = info->prob_lo[d];
    a.dx[d] = info->dx[d];
    a.c[d] = info->ls_center[d];
    a.ub[d] = info->body_u[d];
  }
  a.mask = info->levelset ? 1 : 0;
  a.R = info->ls_radius;
  Stage st;
  if ((rc = st.init((size_t)N * 8))) return rc;
  const std::string root(dir), lev = root + "/Level_0";
  errno = 0;
  if (!make_dir(root) || !make_dir(lev)) return io_fail("ilbm_plotfile_write: cannot create " + lev);
  const std::string dpath = lev + "/Cell_D_00000";
  FILE *fp = std::fopen(dpath.c_str(), "wb");
  if (!fp) return io_fail("ilbm_plotfile_write: cannot create " + dpath);
  FileCloser fc{fp};
  int blo[3], bhi[3];
  for (int d = 0; d < 3; ++d) {
    blo[d] = d < dim ? box->lo[d] : 0;
    bhi[d] = d < dim ? box->hi[d] : 0;
  }
  const std::string fab = "FAB ((8, (64 11 52 0 1 12 0 1023)),(8, (8 7 6 5 4 3 2 1)))" +
                          box_text(dim, blo, bhi) + " " + std::to_string(ncomp) + "\n";
  if (std::fwrite(fab.data(), 1, fab.size(), fp) != fab.size()) return io_fail("plotfile write");
  std::vector<double> vmin(ncomp), vmx(ncomp);
  const double scale = (ctx->storage == ILBM_STORAGE_F16_SCALED)
                           ? (p->f16_scale > 0.0 ? p->f16_scale : 1024.0)
                           : 1.0;
  const int blocks = grid_for(ctx, N);
  const size_t nb = (size_t)N * 8;
  for (int c = 0; c <= ncomp; ++c) {
    if (c < ncomp) {
      const int s = c & 1;
      double *dst = static_cast<double *>(st.d[s]);
      if (c < 6) {
        // rho, ux, uy, uz, vor, Pressure: the scratch planes in that order;
        // a 2D level's uz is the zero of calculateMacroForcing
        const int kind = (c == 0 || c == 5) ? 0 : c;
        const void *src = (c == 3 && dim == 2) ? nullptr : mb + (size_t)c * cs * rb;
        if (rb == 8)
          k_plot_real<double><<<blocks, 256, 0, ctx->stream>>>(a, static_cast<const double *>(src), kind, dst);
        else
          k_plot_real<float><<<blocks, 256, 0, ctx->stream>>>(a, static_cast<const float *>(src), kind, dst);
      } else if (c < 6 + Q) {
        const int q = c - 6;
        const double w = ctx->w[q];
        const char *fb = static_cast<const char *>(box->f_in) + (size_t)q * box->fstride[2] * store_bytes(ctx);
        if (ctx->storage == ILBM_STORAGE_F64)
          k_plot_pop<ILBM_STORAGE_F64><<<blocks, 256, 0, ctx->stream>>>(pf, reinterpret_cast<const double *>(fb), w, 0.0, dst);
        else if (ctx->storage == ILBM_STORAGE_F32_SHIFT)
          k_plot_pop<ILBM_STORAGE_F32_SHIFT><<<blocks, 256, 0, ctx->stream>>>(pf, reinterpret_cast<const float *>(fb), w, 0.0, dst);
        else
          k_plot_pop<ILBM_STORAGE_F16_SCALED><<<blocks, 256, 0, ctx->stream>>>(pf, reinterpret_cast<const __half *>(fb), w, w / scale, dst);
      } else {
        k_plot_phi<<<blocks, 256, 0, ctx->stream>>>(a, dst);
      }
      ctx->launches++;
      cudaMemcpyAsync(st.h[s], st.d[s], nb, cudaMemcpyDeviceToHost, ctx->stream);
      cudaEventRecord(st.ev[s], ctx->stream);
    }
    if (c > 0) {
      const int s = (c - 1) & 1;
      e = cudaEventSynchronize(st.ev[s]);
      if (e != cudaSuccess) return cuda_fail(e, "ilbm_plotfile_write");
      const double *h = static_cast<const double *>(st.h[s]);
      double lo = h[0], hi = h[0];
      for (int64_t t = 1; t < N; ++t) {
        lo = std::min(lo, h[t]);
        hi = std::max(hi, h[t]);
      }
      vmin[c - 1] = lo;
      vmx[c - 1] = hi;
      if (std::fwrite(h, 1, nb, fp) != nb) return io_fail("plotfile write");
    }
  }
  fc.fp = nullptr;
  if (std::fclose(fp) != 0) return io_fail("plotfile write");

  // Level_0/Cell_H: the MultiFab header (one FAB, no ghosts, min / max)
  std::string ch = "1\n1\n" + std::to_string(ncomp) + "\n0\n(1 0\n" + box_text(dim, blo, bhi) +
                   "\n)\n1\nFabOnDisk: Cell_D_00000 0\n\n1," + std::to_string(ncomp) + "\n";
  char buf[64];
  for (int c = 0; c < ncomp; ++c) {
    std::snprintf(buf, sizeof(buf), "%.16e,", vmin[c]);
    ch += buf;
  }
  ch += "\n1," + std::to_string(ncomp) + "\n";
  for (int c = 0; c < ncomp; ++c) {
    std::snprintf(buf, sizeof(buf), "%.16e,", vmx[c]);
    ch += buf;
  }
  ch += "\n";
  errno = 0;
  if (!write_text(lev + "/Cell_H", ch)) return io_fail("plotfile write: Cell_H");

  // Header: variable names, geometry, the level's one grid
  std::string hd = "HyperCLaw-V1.1\n" + std::to_string(ncomp) + "\n";
  const char *mnames[6] = {"rho", "ux", "uy", "uz", "vor", "Pressure"};
  for (int c = 0; c < 6; ++c) hd += std::string(mnames[c]) + "\n";
  for (int q = 0; q < Q; ++q) hd += "f_new_" + std::to_string(q) + "\n";
  if (info->levelset) hd += "phi\n";
  hd += std::to_string(dim) + "\n" + num(info->time) + "\n0\n";
  for (int d = 0; d < dim; ++d) hd += num(info->prob_lo[d]) + " ";
  hd += "\n";
  for (int d = 0; d < dim; ++d) hd += num(info->prob_hi[d]) + " ";
  hd += "\n\n";
  int dlo[3], dhi[3];
  for (int d = 0; d < 3; ++d) {
    dlo[d] = d < dim ? p->domain_lo[d] : 0;
    dhi[d] = d < dim ? p->domain_hi[d] : 0;
  }
  hd += box_text(dim, dlo, dhi) + " \n" + std::to_string(info->istep) + " \n";
  for (int d = 0; d < dim; ++d) hd += num(info->dx[d]) + " ";
  hd += "\n0\n0\n";
  hd += "0 1 " + num(info->time) + "\n" + std::to_string(info->istep) + "\n";
  for (int d = 0; d < dim; ++d) {
    const double glo = info->prob_lo[d] + info->dx[d] * (double)(blo[d] - dlo[d]);
    const double ghi = info->prob_lo[d] + info->dx[d] * (double)(bhi[d] - dlo[d] + 1);
    hd += num(glo) + " " + num(ghi) + "\n";
  }
  hd += "Level_0/Cell\n";
  errno = 0;
  if (!write_text(root + "/Header", hd)) return io_fail("plotfile write: Header");
  return ILBM_OK;
}

}  // extern "C"
