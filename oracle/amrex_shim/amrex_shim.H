// Minimal AMReX-compatible shim: TEST INFRASTRUCTURE ONLY.
//
// It lets the reference's own per-cell headers (Source/LBM/*.H,
// Source/BC/bc_fill.H, bc_val.H), its marker immersed-boundary backend
// (Source/IBM/IBMarkerDF.cpp), its force evaluator (Source/IBM/IBForceEval.cpp)
// and the example problem hooks (Examples/*/Prob.H,
// Examples/Pitching_airfoil/IBMUserDefinedGeometry.H) compile unchanged, in
// place, on the host, so the oracle can be checked against them.
//
// Scope: one box per level, one rank, serial host loops.  Every type here is
// written for this project; nothing is taken from AMReX.  Semantics follow
// AMReX's public documentation for the few operations the reference uses:
//   * Array4 component-major indexing over the allocated (grown) box;
//   * MultiFab::FillBoundary(periodicity): ghost cells whose periodic image is
//     a valid cell receive that cell's value;
//   * MultiFab::SumBoundary(periodicity): ghost-cell values are added into the
//     valid cells they overlap (periodic images included), ghosts unchanged;
//   * ParticleContainer::Redistribute: single tile, positions wrapped in
//     periodic directions, order preserved.
// The product never includes this file.
#pragma once

#ifndef AMREX_SPACEDIM
#error "compile with -DAMREX_SPACEDIM=2 or 3"
#endif

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#ifndef AMREX_PARTICLES
#define AMREX_PARTICLES 1
#endif

#define AMREX_GPU_HOST_DEVICE
#define AMREX_GPU_DEVICE
#define AMREX_GPU_HOST
#define AMREX_FORCE_INLINE inline
#define AMREX_INLINE inline
#define AMREX_USE_GPU_PRINTF_SHIM 1

#if (AMREX_SPACEDIM == 2)
#define AMREX_D_TERM(a, b, c) a b
#define AMREX_D_DECL(a, b, c) a, b
#else
#define AMREX_D_TERM(a, b, c) a b c
#define AMREX_D_DECL(a, b, c) a, b, c
#endif

#define AMREX_ALWAYS_ASSERT(x)                                                  \
  do {                                                                         \
    if (!(x)) ::amrex::Abort("assertion failed: " #x);                         \
  } while (0)
#define AMREX_ALWAYS_ASSERT_WITH_MESSAGE(x, m)                                  \
  do {                                                                         \
    if (!(x)) ::amrex::Abort(m);                                               \
  } while (0)
#define AMREX_ASSERT(x) ((void)0)
#define BL_ASSERT(x) ((void)0)
#define BL_PROFILE(x) ((void)0)

namespace amrex {

#ifdef SHIM_REAL_FLOAT
using Real = float;
#else
using Real = double;
#endif
using ParticleReal = Real;
using Long = long long;

template <class T>
using Vector = std::vector<T>;

[[noreturn]] inline void Abort(const std::string &msg = "") {
  throw std::runtime_error("amrex::Abort: " + msg);
}

template <class... Ts>
inline void ignore_unused(const Ts &...) {}

template <class T>
constexpr T max(T a, T b) { return (a < b) ? b : a; }
template <class T>
constexpr T min(T a, T b) { return (b < a) ? b : a; }

template <class T, int N>
struct GpuArray {
  T arr[N];
  T &operator[](int i) { return arr[i]; }
  const T &operator[](int i) const { return arr[i]; }
  T *data() { return arr; }
  const T *data() const { return arr; }
  static constexpr int size() { return N; }
  T *begin() { return arr; }
  T *end() { return arr + N; }
};

template <class T, std::size_t N>
using Array = std::array<T, N>;

struct IntVect {
  int vect[AMREX_SPACEDIM];
  IntVect() { for (int d = 0; d < AMREX_SPACEDIM; ++d) vect[d] = 0; }
#if (AMREX_SPACEDIM == 2)
  IntVect(int i, int j) { vect[0] = i; vect[1] = j; }
#else
  IntVect(int i, int j, int k) { vect[0] = i; vect[1] = j; vect[2] = k; }
#endif
  explicit IntVect(int s) { for (int d = 0; d < AMREX_SPACEDIM; ++d) vect[d] = s; }
  int &operator[](int d) { return vect[d]; }
  const int &operator[](int d) const { return vect[d]; }
  static IntVect TheZeroVector() { return IntVect(0); }
};

struct Box {
  IntVect smallend, bigend;
  Box() : smallend(0), bigend(-1) {}
  Box(const IntVect &lo, const IntVect &hi) : smallend(lo), bigend(hi) {}
  int smallEnd(int d) const { return smallend[d]; }
  int bigEnd(int d) const { return bigend[d]; }
  const IntVect &smallEnd() const { return smallend; }
  const IntVect &bigEnd() const { return bigend; }
  const int *loVect() const { return smallend.vect; }
  const int *hiVect() const { return bigend.vect; }
  bool ok() const {
    for (int d = 0; d < AMREX_SPACEDIM; ++d)
      if (bigend[d] < smallend[d]) return false;
    return true;
  }
  bool contains(const IntVect &iv) const {
    for (int d = 0; d < AMREX_SPACEDIM; ++d)
      if (iv[d] < smallend[d] || iv[d] > bigend[d]) return false;
    return true;
  }
  bool contains(int i, int j, int k) const {
#if (AMREX_SPACEDIM == 2)
    (void)k;
    return contains(IntVect(i, j));
#else
    return contains(IntVect(i, j, k));
#endif
  }
  bool contains(const Box &b) const {
    return contains(b.smallend) && contains(b.bigend);
  }
  IntVect length() const {
    IntVect l;
    for (int d = 0; d < AMREX_SPACEDIM; ++d) l[d] = bigend[d] - smallend[d] + 1;
    return l;
  }
  Long numPts() const {
    if (!ok()) return 0;
    Long n = 1;
    for (int d = 0; d < AMREX_SPACEDIM; ++d) n *= (bigend[d] - smallend[d] + 1);
    return n;
  }
  Box &operator&=(const Box &b) {
    for (int d = 0; d < AMREX_SPACEDIM; ++d) {
      smallend[d] = std::max(smallend[d], b.smallend[d]);
      bigend[d] = std::min(bigend[d], b.bigend[d]);
    }
    return *this;
  }
  Box &grow(int n) {
    for (int d = 0; d < AMREX_SPACEDIM; ++d) { smallend[d] -= n; bigend[d] += n; }
    return *this;
  }
  Box &grow(int d, int n) { smallend[d] -= n; bigend[d] += n; return *this; }
};
inline Box operator&(Box a, const Box &b) { a &= b; return a; }
inline Box grow(Box b, int n) { return b.grow(n); }

template <class T>
struct Array4 {
  T *p = nullptr;
  Long jstride = 0, kstride = 0, nstride = 0;
  int b0 = 0, b1 = 0, b2 = 0;
  int ncomp = 0;
  Array4() = default;
  Array4(T *ptr, const Box &gbox, int nc) : p(ptr), ncomp(nc) {
    const IntVect len = gbox.length();
    b0 = gbox.smallEnd(0);
    b1 = gbox.smallEnd(1);
#if (AMREX_SPACEDIM == 3)
    b2 = gbox.smallEnd(2);
    jstride = len[0];
    kstride = (Long)len[0] * len[1];
    nstride = kstride * len[2];
#else
    b2 = 0;
    jstride = len[0];
    kstride = (Long)len[0] * len[1];
    nstride = kstride;
#endif
  }
  template <class U>
  Array4(const Array4<U> &o)
      : p(o.p), jstride(o.jstride), kstride(o.kstride), nstride(o.nstride),
        b0(o.b0), b1(o.b1), b2(o.b2), ncomp(o.ncomp) {}
  Long off(int i, int j, int k) const {
    return (Long)(i - b0) + (Long)(j - b1) * jstride + (Long)(k - b2) * kstride;
  }
  T &operator()(int i, int j, int k) const { return p[off(i, j, k)]; }
  T &operator()(int i, int j, int k, int n) const {
    return p[off(i, j, k) + (Long)n * nstride];
  }
  T &operator()(const IntVect &iv, int n) const {
#if (AMREX_SPACEDIM == 2)
    return (*this)(iv[0], iv[1], 0, n);
#else
    return (*this)(iv[0], iv[1], iv[2], n);
#endif
  }
  T &operator()(const IntVect &iv) const { return (*this)(iv, 0); }
  int nComp() const { return ncomp; }
};

namespace BCType {
enum mathematicalBndryTypes : int {
  bogus = -666,
  reflect_odd = -1,
  int_dir = 0,
  reflect_even = 1,
  foextrap = 2,
  ext_dir = 3,
  hoextrap = 4,
  user_1 = 1001,
  user_2 = 1002,
  user_3 = 1003
};
}

struct BCRec {
  int bc_lo[AMREX_SPACEDIM];
  int bc_hi[AMREX_SPACEDIM];
  BCRec() {
    for (int d = 0; d < AMREX_SPACEDIM; ++d) bc_lo[d] = bc_hi[d] = BCType::bogus;
  }
  int lo(int d) const { return bc_lo[d]; }
  int hi(int d) const { return bc_hi[d]; }
  void setLo(int d, int v) { bc_lo[d] = v; }
  void setHi(int d, int v) { bc_hi[d] = v; }
};

struct Periodicity {
  int period[AMREX_SPACEDIM];
  bool isAnyPeriodic() const {
    for (int d = 0; d < AMREX_SPACEDIM; ++d)
      if (period[d] > 0) return true;
    return false;
  }
};

struct GeometryData {
  Box domain;
  Real prob_lo[AMREX_SPACEDIM];
  Real prob_hi[AMREX_SPACEDIM];
  Real dx[AMREX_SPACEDIM];
  int is_periodic[AMREX_SPACEDIM];
  const Box &Domain() const { return domain; }
  const Real *CellSize() const { return dx; }
  const Real *ProbLo() const { return prob_lo; }
  int isPeriodic(int d) const { return is_periodic[d]; }
};

class Geometry {
 public:
  Geometry() = default;
  Geometry(const Box &dom, const Real *plo, const Real *phi, const int *per) {
    gd.domain = dom;
    for (int d = 0; d < AMREX_SPACEDIM; ++d) {
      gd.prob_lo[d] = plo[d];
      gd.prob_hi[d] = phi[d];
      gd.dx[d] = (phi[d] - plo[d]) / Real(dom.bigEnd(d) - dom.smallEnd(d) + 1);
      gd.is_periodic[d] = per[d];
    }
  }
  GpuArray<Real, AMREX_SPACEDIM> CellSizeArray() const {
    GpuArray<Real, AMREX_SPACEDIM> a;
    for (int d = 0; d < AMREX_SPACEDIM; ++d) a[d] = gd.dx[d];
    return a;
  }
  GpuArray<Real, AMREX_SPACEDIM> ProbLoArray() const {
    GpuArray<Real, AMREX_SPACEDIM> a;
    for (int d = 0; d < AMREX_SPACEDIM; ++d) a[d] = gd.prob_lo[d];
    return a;
  }
  GpuArray<Real, AMREX_SPACEDIM> ProbHiArray() const {
    GpuArray<Real, AMREX_SPACEDIM> a;
    for (int d = 0; d < AMREX_SPACEDIM; ++d) a[d] = gd.prob_hi[d];
    return a;
  }
  Real CellSize(int d) const { return (d < AMREX_SPACEDIM) ? gd.dx[d] : Real(0); }
  Real ProbLo(int d) const { return gd.prob_lo[d]; }
  Real ProbHi(int d) const { return gd.prob_hi[d]; }
  const Box &Domain() const { return gd.domain; }
  bool isPeriodic(int d) const { return gd.is_periodic[d] != 0; }
  bool isAllPeriodic() const {
    for (int d = 0; d < AMREX_SPACEDIM; ++d)
      if (!gd.is_periodic[d]) return false;
    return true;
  }
  GpuArray<int, AMREX_SPACEDIM> isPeriodicArray() const {
    GpuArray<int, AMREX_SPACEDIM> a;
    for (int d = 0; d < AMREX_SPACEDIM; ++d) a[d] = gd.is_periodic[d];
    return a;
  }
  Periodicity periodicity() const {
    Periodicity p;
    for (int d = 0; d < AMREX_SPACEDIM; ++d)
      p.period[d] = gd.is_periodic[d] ? (gd.domain.bigEnd(d) - gd.domain.smallEnd(d) + 1) : 0;
    return p;
  }
  const GeometryData &data() const { return gd; }

 private:
  GeometryData gd;
};

struct BoxArray {
  std::vector<Box> boxes;
  BoxArray() = default;
  explicit BoxArray(const Box &b) : boxes(1, b) {}
  int size() const { return (int)boxes.size(); }
  const Box &operator[](int i) const { return boxes[i]; }
};
struct DistributionMapping {};
inline bool operator!=(const BoxArray &a, const BoxArray &b) {
  if (a.size() != b.size()) return true;
  for (int n = 0; n < a.size(); ++n)
    for (int d = 0; d < AMREX_SPACEDIM; ++d)
      if (a[n].smallEnd(d) != b[n].smallEnd(d) || a[n].bigEnd(d) != b[n].bigEnd(d)) return true;
  return false;
}
inline bool operator!=(const DistributionMapping &, const DistributionMapping &) { return false; }

struct FArrayBox {
  Box gbox;
  int nc = 0;
  std::vector<Real> data;
  FArrayBox() = default;
  FArrayBox(const Box &b, int n) : gbox(b), nc(n), data((size_t)b.numPts() * n, Real(0)) {}
  const Box &box() const { return gbox; }
  int nComp() const { return nc; }
  Array4<Real> array() { return Array4<Real>(data.data(), gbox, nc); }
  Array4<Real> array(int n) {
    Array4<Real> a(data.data(), gbox, nc);
    a.p += (Long)n * a.nstride;
    a.ncomp = nc - n;
    return a;
  }
  Array4<const Real> array() const { return Array4<const Real>(data.data(), gbox, nc); }
  Array4<const Real> const_array() const { return array(); }
  Array4<const Real> const_array(int n) const {
    Array4<const Real> a(data.data(), gbox, nc);
    a.p += (Long)n * a.nstride;
    a.ncomp = nc - n;
    return a;
  }
};

class MultiFab;

class MFIter {
 public:
  MFIter(const MultiFab &mf, bool tiling = false);
  bool isValid() const { return idx < nfab; }
  MFIter &operator++() { ++idx; return *this; }
  int index() const { return idx; }
  Box validbox() const;
  Box tilebox() const { return validbox(); }
  Box fabbox() const;
  Box growntilebox(int n) const;

 private:
  const MultiFab *m;
  int idx = 0;
  int nfab = 0;
};

inline bool TilingIfNotGPU() { return false; }

enum MakeType { make_alias = 0 };

class MultiFab {
 public:
  MultiFab() = default;
  MultiFab(const BoxArray &ba_, const DistributionMapping &, int ncomp, int ngrow)
      : ba(ba_), nc(ncomp), ng(ngrow) {
    for (const Box &b : ba.boxes) {
      Box g = b;
      g.grow(ngrow);
      fabs.emplace_back(g, ncomp);
    }
  }
  int nComp() const { return nc; }
  int nGrow() const { return ng; }
  bool ok() const { return !fabs.empty(); }
  const BoxArray &boxArray() const { return ba; }
  DistributionMapping DistributionMap() const { return {}; }
  int size() const { return (int)fabs.size(); }
  FArrayBox &operator[](int i) { return fabs[i]; }
  const FArrayBox &operator[](int i) const { return fabs[i]; }
  template <class It>
  FArrayBox &operator[](const It &it) { return fabs[it.index()]; }
  template <class It>
  const FArrayBox &operator[](const It &it) const { return fabs[it.index()]; }

  void setVal(Real v) {
    for (auto &f : fabs) std::fill(f.data.begin(), f.data.end(), v);
  }

  // Ghost cells whose periodic image lies in a valid box receive that value.
  void FillBoundary(const Periodicity &per) { FillBoundary(0, nc, per); }
  void FillBoundary(int scomp, int ncomp, const Periodicity &per) {
    forEachGhostImage(per, [&](FArrayBox &dst, const IntVect &g, FArrayBox &src, const IntVect &v) {
      auto d = dst.array();
      auto s = src.array();
      for (int n = scomp; n < scomp + ncomp; ++n) d(g, n) = s(v, n);
    });
  }
  // Ghost values are added into the valid cells they overlap; ghosts keep their values.
  void SumBoundary(int scomp, int ncomp, const Periodicity &per) {
    std::vector<std::vector<Real>> snap;
    for (auto &f : fabs) snap.push_back(f.data);
    forEachGhostImage(per, [&](FArrayBox &dst, const IntVect &g, FArrayBox &src, const IntVect &v) {
      const size_t di = &dst - fabs.data();
      Array4<Real> gs(snap[di].data(), dst.gbox, nc);
      auto s = src.array();
      for (int n = scomp; n < scomp + ncomp; ++n) s(v, n) += gs(g, n);
    });
  }
  void SumBoundary(const Periodicity &per) { SumBoundary(0, nc, per); }

  static void Saxpy(MultiFab &dst, Real a, const MultiFab &src, int scomp, int dcomp,
                    int ncomp, int nghost) {
    for (int f = 0; f < dst.size(); ++f) {
      Box b = dst.ba[f];
      b.grow(nghost);
      auto d = dst.fabs[f].array();
      auto s = src.fabs[f].const_array();
      forBox(b, [&](const IntVect &iv) {
        for (int n = 0; n < ncomp; ++n) d(iv, dcomp + n) += a * s(iv, scomp + n);
      });
    }
  }
  static void Add(MultiFab &dst, const MultiFab &src, int scomp, int dcomp, int ncomp,
                  int nghost) {
    for (int f = 0; f < dst.size(); ++f) {
      Box b = dst.ba[f];
      b.grow(nghost);
      auto d = dst.fabs[f].array();
      auto s = src.fabs[f].const_array();
      forBox(b, [&](const IntVect &iv) {
        for (int n = 0; n < ncomp; ++n) d(iv, dcomp + n) += s(iv, scomp + n);
      });
    }
  }
  static void Copy(MultiFab &dst, const MultiFab &src, int scomp, int dcomp, int ncomp,
                   int nghost) {
    for (int f = 0; f < dst.size(); ++f) {
      Box b = dst.ba[f];
      b.grow(nghost);
      auto d = dst.fabs[f].array();
      auto s = src.fabs[f].const_array();
      forBox(b, [&](const IntVect &iv) {
        for (int n = 0; n < ncomp; ++n) d(iv, dcomp + n) = s(iv, scomp + n);
      });
    }
  }
  template <class F>
  static void forBox(const Box &b, F &&fn) {
#if (AMREX_SPACEDIM == 3)
    for (int k = b.smallEnd(2); k <= b.bigEnd(2); ++k)
#endif
      for (int j = b.smallEnd(1); j <= b.bigEnd(1); ++j)
        for (int i = b.smallEnd(0); i <= b.bigEnd(0); ++i) {
#if (AMREX_SPACEDIM == 3)
          fn(IntVect(i, j, k));
#else
          fn(IntVect(i, j));
#endif
        }
  }

  BoxArray ba;
  int nc = 0, ng = 0;
  std::vector<FArrayBox> fabs;

 private:
  // Visits only the ghost cells of each fab (rows inside the valid box touch
  // just their ghost columns), so large boxes stay cheap.
 public:
  template <class F>
  static void forGhost(const Box &gb, const Box &vb, F &&fn) {
#if (AMREX_SPACEDIM == 3)
    for (int k = gb.smallEnd(2); k <= gb.bigEnd(2); ++k)
#else
    const int k = 0;
#endif
      for (int j = gb.smallEnd(1); j <= gb.bigEnd(1); ++j) {
        bool row_in = (j >= vb.smallEnd(1) && j <= vb.bigEnd(1));
#if (AMREX_SPACEDIM == 3)
        row_in = row_in && (k >= vb.smallEnd(2) && k <= vb.bigEnd(2));
#endif
        for (int i = gb.smallEnd(0); i <= gb.bigEnd(0); ++i) {
          if (row_in && i == vb.smallEnd(0)) i = vb.bigEnd(0) + 1;
          if (i > gb.bigEnd(0)) break;
#if (AMREX_SPACEDIM == 3)
          fn(IntVect(i, j, k));
#else
          (void)k;
          fn(IntVect(i, j));
#endif
        }
      }
  }

  template <class F>
  void forEachGhostImage(const Periodicity &per, F &&fn) {
    for (auto &dst : fabs) {
      const size_t di0 = &dst - fabs.data();
      forGhost(dst.gbox, ba[(int)di0], [&](const IntVect &g) {
        const size_t di = di0;
        // try every periodic shift (including zero) onto every valid box
        int sh[3][3];
        int nsh[3];
        for (int d = 0; d < 3; ++d) { nsh[d] = 1; sh[d][0] = 0; }
        for (int d = 0; d < AMREX_SPACEDIM; ++d) {
          if (per.period[d] > 0) {
            nsh[d] = 3;
            sh[d][1] = per.period[d];
            sh[d][2] = -per.period[d];
          }
        }
        for (int a = 0; a < nsh[0]; ++a)
          for (int b = 0; b < nsh[1]; ++b)
            for (int c = 0; c < nsh[2]; ++c) {
              IntVect v = g;
              v[0] += sh[0][a];
              v[1] += sh[1][b];
#if (AMREX_SPACEDIM == 3)
              v[2] += sh[2][c];
#else
              if (c > 0) continue;
#endif
              for (int s = 0; s < (int)fabs.size(); ++s) {
                if (s == (int)di && a == 0 && b == 0 && c == 0) continue;
                if (ba[s].contains(v)) fn(dst, g, fabs[s], v);
              }
            }
      });
    }
  }
};

inline MFIter::MFIter(const MultiFab &mf, bool) : m(&mf), idx(0), nfab(mf.size()) {}
inline Box MFIter::validbox() const { return m->boxArray()[idx]; }
inline Box MFIter::fabbox() const { return (*m)[idx].box(); }
inline Box MFIter::growntilebox(int n) const {
  Box b = validbox();
  b.grow(n);
  return b & fabbox();
}

template <class F>
inline void ParallelFor(Long n, F &&f) {
  for (Long i = 0; i < n; ++i) f((int)i);
}
template <class F>
inline void ParallelFor(int n, F &&f) {
  for (int i = 0; i < n; ++i) f(i);
}
template <class F>
inline void ParallelFor(const Box &b, F &&f) {
#if (AMREX_SPACEDIM == 3)
  for (int k = b.smallEnd(2); k <= b.bigEnd(2); ++k)
#else
  const int k = 0;
#endif
    for (int j = b.smallEnd(1); j <= b.bigEnd(1); ++j)
      for (int i = b.smallEnd(0); i <= b.bigEnd(0); ++i) f(i, j, k);
}
template <class F>
inline void Loop(const Box &b, F &&f) { ParallelFor(b, f); }

namespace Gpu {
template <class T>
using DeviceVector = std::vector<T>;
struct HostToDevice {};
struct DeviceToHost {};
static constexpr HostToDevice hostToDevice{};
static constexpr DeviceToHost deviceToHost{};
template <class Tag, class InIt, class OutIt>
inline void copy(Tag, InIt first, InIt last, OutIt dest) { std::copy(first, last, dest); }
inline bool notInLaunchRegion() { return true; }
namespace Atomic {
template <class T>
inline void AddNoRet(T *p, T v) { *p += v; }
template <class T>
inline T Add(T *p, T v) { T o = *p; *p += v; return o; }
}  // namespace Atomic
}  // namespace Gpu

namespace ParallelDescriptor {
inline int MyProc() { return 0; }
inline int IOProcessorNumber() { return 0; }
inline bool IOProcessor() { return true; }
inline int NProcs() { return 1; }
template <class T>
inline void ReduceRealSum(T &) {}
template <class T>
inline void ReduceRealMin(T &) {}
template <class T>
inline void ReduceRealMax(T &) {}
template <class T>
inline void ReduceLongSum(T &) {}
}  // namespace ParallelDescriptor

class Print {
 public:
  Print() = default;
  ~Print() {
    if (std::getenv("ILBM_SHIM_VERBOSE")) std::cerr << ss.str();
  }
  template <class T>
  Print &operator<<(const T &v) { ss << v; return *this; }
  Print &operator<<(std::ostream &(*f)(std::ostream &)) { f(ss); return *this; }
  Print &operator<<(std::ios_base &(*f)(std::ios_base &)) { f(ss); return *this; }

 private:
  std::ostringstream ss;
};

namespace Math {
template <class T>
inline T abs(T x) { return std::abs(x); }
template <class T>
constexpr T pi() { return T(3.14159265358979323846264338327950288); }
template <int N, class T>
inline T powi(T x) {
  T r = T(1);
  for (int i = 0; i < N; ++i) r *= x;
  return r;
}
template <class T>
inline T floor(T x) { return std::floor(x); }
template <class T>
inline std::pair<T, T> sincos(T x) { return {std::sin(x), std::cos(x)}; }
}  // namespace Math

// ----------------------------------------------------------------------------
// Particles: one tile (grid 0, tile 0) on one rank.
// ----------------------------------------------------------------------------
template <int NArrayReal, int NArrayInt>
struct ShimParticle {
  Real m_pos[AMREX_SPACEDIM];
  Long m_id = 0;
  int m_cpu = 0;
  Real &pos(int d) { return m_pos[d]; }
  const Real &pos(int d) const { return m_pos[d]; }
  Long &id() { return m_id; }
  Long id() const { return m_id; }
  int &cpu() { return m_cpu; }
};

template <int NArrayReal, int NArrayInt>
struct ShimSoA {
  std::vector<ParticleReal> real[NArrayReal];
  std::vector<int> ints[NArrayInt > 0 ? NArrayInt : 1];
  std::vector<ParticleReal> &GetRealData(int i) { return real[i]; }
  const std::vector<ParticleReal> &GetRealData(int i) const { return real[i]; }
  std::vector<int> &GetIntData(int i) { return ints[i]; }
  const std::vector<int> &GetIntData(int i) const { return ints[i]; }
};

template <int NArrayReal, int NArrayInt>
struct ShimParticleTile {
  using ParticleType = ShimParticle<NArrayReal, NArrayInt>;
  std::vector<ParticleType> aos;
  ShimSoA<NArrayReal, NArrayInt> soa;
  void push_back(const ParticleType &p) { aos.push_back(p); }
  void push_back_real(const std::array<ParticleReal, NArrayReal> &a) {
    for (int i = 0; i < NArrayReal; ++i) soa.real[i].push_back(a[i]);
  }
  void push_back_int(const std::array<int, NArrayInt> &a) {
    for (int i = 0; i < NArrayInt; ++i) soa.ints[i].push_back(a[i]);
  }
  Long numParticles() const { return (Long)aos.size(); }
  std::vector<ParticleType> &GetArrayOfStructs() { return aos; }
  const std::vector<ParticleType> &GetArrayOfStructs() const { return aos; }
  ShimSoA<NArrayReal, NArrayInt> &GetStructOfArrays() { return soa; }
  const ShimSoA<NArrayReal, NArrayInt> &GetStructOfArrays() const { return soa; }
};

template <int NStructReal, int NStructInt, int NArrayReal, int NArrayInt>
class ParticleContainer {
 public:
  using ParticleType = ShimParticle<NArrayReal, NArrayInt>;
  using ParticleTileType = ShimParticleTile<NArrayReal, NArrayInt>;
  using Tiles = std::map<std::pair<int, int>, ParticleTileType>;

  ParticleContainer(const Geometry &g, const DistributionMapping &, const BoxArray &)
      : geom(g) {}
  Tiles &GetParticles(int) { return tiles; }
  void Redistribute() {
    for (auto &kv : tiles) {
      for (auto &p : kv.second.aos) {
        for (int d = 0; d < AMREX_SPACEDIM; ++d) {
          if (!geom.isPeriodic(d)) continue;
          const Real lo = geom.ProbLo(d), hi = geom.ProbHi(d), L = hi - lo;
          while (p.m_pos[d] < lo) p.m_pos[d] += L;
          while (p.m_pos[d] >= hi) p.m_pos[d] -= L;
        }
      }
    }
  }
  Long TotalNumberOfParticles() const {
    Long n = 0;
    for (auto &kv : tiles) n += kv.second.numParticles();
    return n;
  }

  Geometry geom;
  Tiles tiles;
};

template <int NStructReal, int NStructInt, int NArrayReal, int NArrayInt>
class ParIter {
 public:
  using PC = ParticleContainer<NStructReal, NStructInt, NArrayReal, NArrayInt>;
  ParIter(PC &pc, int) : it(pc.tiles.begin()), end(pc.tiles.end()) {}
  bool isValid() const { return it != end; }
  ParIter &operator++() { ++it; return *this; }
  int index() const { return it->first.first; }
  Long numParticles() const { return it->second.numParticles(); }
  auto &GetArrayOfStructs() { return it->second.aos; }
  auto &GetStructOfArrays() { return it->second.soa; }
  auto &GetParticleTile() { return it->second; }

 private:
  typename PC::Tiles::iterator it, end;
};

}  // namespace amrex
