// Reference CPU build ("refcpu"): TEST INFRASTRUCTURE ONLY.
//
// This translation unit compiles the reference's own sources, unchanged and
// in place under the reference tree, against the project-written shim in
// oracle/amrex_shim/:
//   Source/LBM/feq.H, collide.H, collide_forced.H, stream.H,
//   calculateMacroForcing.H          per-cell LBM arithmetic
//   Source/BC/bc_fill.H, bc_val.{H,cpp}  ghost-cell functors (mesoscopicBcFill,
//                                        macroBcFill)
//   Source/IBM/IBMarkerDF.cpp        the whole marker direct-forcing IBM
//                                    (markers, delta kernels, explicit/diag/IVC
//                                    force, spreading, export)
//   Source/IBM/IBForceEval.cpp       link-wise momentum exchange
//   Examples/Pitching_airfoil/IBMUserDefinedGeometry.H  (2D builds, when on
//                                    the include path) NACA marker hook
//
// Around them it restates, for ONE level held in ONE box, the parts of the
// level advance that live in files which need the full AMReX runtime:
//   AmrCoreLBM::AdvancePhiAtLevel     Source/Core/AdvanceLBMAtLevel.cpp:20-394
//   FillPatchSingleLevel + PhysBCFunct (AMReX; documented semantics: copy of
//     valid + periodic images, then per ghost cell the built-in foextrap fill
//     followed by the user functor, faces before edges before corners)
//   AmrCoreLBM::InitEquilibrium       Source/Core/AmrCoreLBM.cpp:2117-2164
//   AmrCoreLBM::ComputeIBForce        Source/Core/AmrCoreLBM.cpp:456-631
//   tau/dt rules                      Source/Core/AmrCoreLBM.cpp:225-238
//
// The pass structure (FillPatch copies, collide, FillBoundary, bounce-back,
// stream, macro) is kept as in the reference so this build also serves as the
// timed CPU baseline; the box passes use OpenMP over the outer loop.
// It is a checker and a baseline, never part of the product.

#include <feq.H>
#include <collide.H>
#include <collide_forced.H>
#include <stream.H>
#include <calculateMacroForcing.H>
#include <bc_fill.H>
#include "BC/bc_val.cpp"
#include "IBM/IBMarkerDF.cpp"
#include "IBM/IBForceEval.cpp"
#include "LevelSet/LevelSet.cpp"
#include <visPara.H>
#include <Tagging.H>

#include "oracle_case.h"

#ifdef _OPENMP
#include <omp.h>
#endif

#include <cstring>

namespace {
using namespace amrex;

#if (AMREX_SPACEDIM == 3)
#define REF_IV(i, j, k) IntVect(i, j, k)
#else
#define REF_IV(i, j, k) IntVect(i, j)
#endif

struct RefLevel {
  ilbm_case c;
  int ndir = 0;
  Vector<Real> wi, dirx, diry, dirz;
  Geometry geom;
  BoxArray ba;
  DistributionMapping dm;
  int nghost = 3;
  int nmac = 6;
  MultiFab f_new, f_old, macro_new, macro_old, forcing;
  BCBuf bcval;
  std::vector<BCRec> bcsMeso, bcsMacro;
  Real tau = 0, dt = 0;
  Real time = 0;
  long step = 0;
  std::unique_ptr<IBMarkerDF> ibm;
  ilbm_ib_case ibc;
  bool use_ib = false;
  bool have_prev = false;
  Real prev_body[3] = {0, 0, 0};
  double rec[ILBM_FORCE_REC];
  MultiFab last_fx;  // fx_cc/fy_cc/fz_cc of the last step (valid cells)
  // per-step scratch of AdvancePhiAtLevel (:43-60); kept allocated between
  // steps the way AMReX's arena recycles them
  MultiFab fx_cc, fy_cc, fz_cc, sfS, smS;
};

template <class F>
void for_box(const Box &b, F &&fn) {
#if (AMREX_SPACEDIM == 3)
#pragma omp parallel for schedule(static)
  for (int k = b.smallEnd(2); k <= b.bigEnd(2); ++k)
    for (int j = b.smallEnd(1); j <= b.bigEnd(1); ++j)
      for (int i = b.smallEnd(0); i <= b.bigEnd(0); ++i) fn(i, j, k);
#else
#pragma omp parallel for schedule(static)
  for (int j = b.smallEnd(1); j <= b.bigEnd(1); ++j)
    for (int i = b.smallEnd(0); i <= b.bigEnd(0); ++i) fn(i, j, 0);
#endif
}

// AMReX built-in first-order extrapolation for one ghost cell (the only
// built-in physical BC the reference decks use besides the user functors).
void filcc_cell(const IntVect &iv, Array4<Real> const &q, int ncomp, const Box &dom,
                const BCRec *bcr) {
  for (int n = 0; n < ncomp; ++n) {
    const BCRec &bc = bcr[n];
    for (int d = 0; d < AMREX_SPACEDIM; ++d) {
      IntVect src = iv;
      int code = -12345;
      if (iv[d] < dom.smallEnd(d)) {
        code = bc.lo(d);
        src[d] = dom.smallEnd(d);
      } else if (iv[d] > dom.bigEnd(d)) {
        code = bc.hi(d);
        src[d] = dom.bigEnd(d);
      } else {
        continue;
      }
      if (code == BCType::foextrap) {
        q(iv, n) = q(src, n);
      } else if (code == BCType::hoextrap || code == BCType::reflect_even ||
                 code == BCType::reflect_odd) {
        Abort("refcpu: unsupported built-in BC type");
      }
    }
  }
}

// FillPatchSingleLevel(dst <- src) with PhysBCFunct<GpuBndryFuncFab<F>>.
template <class UserF>
void fill_patch(RefLevel &L, MultiFab &dst, const MultiFab &src, int ncomp,
                const std::vector<BCRec> &bcs, const UserF &user) {
  const Box vb = L.ba[0];
  {
    auto d = dst[0].array();
    auto s = src[0].const_array();
    for_box(vb, [&](int i, int j, int k) {
      for (int n = 0; n < ncomp; ++n) d(i, j, k, n) = s(i, j, k, n);
    });
  }
  dst.FillBoundary(0, ncomp, L.geom.periodicity());

  const Box &dom = L.geom.Domain();
  const Box gb = dst[0].box();
  Box gdom = dom;
  for (int d = 0; d < AMREX_SPACEDIM; ++d)
    if (L.geom.isPeriodic(d)) gdom.grow(d, L.nghost + 1);
  if (gdom.contains(gb)) return;
  auto a = dst[0].array();
  const GeometryData gd = L.geom.data();
  for (int cls = 1; cls <= AMREX_SPACEDIM; ++cls) {
    MultiFab::forGhost(gb, dom, [&](const IntVect &iv) {
      int nout = 0;
      for (int d = 0; d < AMREX_SPACEDIM; ++d)
        if (iv[d] < gdom.smallEnd(d) || iv[d] > gdom.bigEnd(d)) ++nout;
      if (nout != cls) return;
      filcc_cell(iv, a, ncomp, dom, bcs.data());
      user(iv, a, 0, ncomp, gd, L.time, bcs.data(), 0, 0);
    });
  }
}

void build_level(RefLevel &L, const ilbm_case &c) {
  if (c.dim != AMREX_SPACEDIM) Abort("refcpu: case dimension does not match this build");
  L.c = c;
  L.ndir = c.q;
  if (L.ndir > BCBuf::MAX_NDIR) Abort("LBM ndir exceeds BCBuf::MAX_NDIR (27).");
  L.wi.resize(L.ndir);
  L.dirx.resize(L.ndir);
  L.diry.resize(L.ndir);
  L.dirz.resize(L.ndir);
  for (int q = 0; q < L.ndir; ++q) {
    L.wi[q] = Real(c.wis[q]) / Real(c.wim[q]);  // AmrCoreLBM.cpp:1218-1221
    L.dirx[q] = Real(c.cx[q]);
    L.diry[q] = Real(c.cy[q]);
    L.dirz[q] = Real(c.cz[q]);
  }
  L.nghost = c.nghost > 0 ? c.nghost : 3;
  IntVect lo(0), hi(0);
  Real plo[AMREX_SPACEDIM], phi[AMREX_SPACEDIM];
  int per[AMREX_SPACEDIM];
  for (int d = 0; d < AMREX_SPACEDIM; ++d) {
    hi[d] = c.n_cell[d] - 1;
    plo[d] = Real(c.prob_lo[d]);
    phi[d] = Real(c.prob_hi[d]);
    per[d] = c.periodic[d];
  }
  Box dom(lo, hi);
  L.geom = Geometry(dom, plo, phi, per);
  L.ba = BoxArray(dom);
  L.f_new = MultiFab(L.ba, L.dm, L.ndir, L.nghost);
  L.f_old = MultiFab(L.ba, L.dm, L.ndir, L.nghost);
  L.macro_new = MultiFab(L.ba, L.dm, L.nmac, L.nghost);
  L.macro_old = MultiFab(L.ba, L.dm, L.nmac, L.nghost);
  L.forcing = MultiFab(L.ba, L.dm, 3, L.nghost);
  L.last_fx = MultiFab(L.ba, L.dm, 3, 0);
  L.fx_cc = MultiFab(L.ba, L.dm, 1, L.nghost);
  L.fy_cc = MultiFab(L.ba, L.dm, 1, L.nghost);
  L.fz_cc = MultiFab(L.ba, L.dm, 1, L.nghost);
  L.sfS = MultiFab(L.ba, L.dm, L.ndir, L.nghost);
  L.smS = MultiFab(L.ba, L.dm, L.nmac, L.nghost);

  // AmrCoreLBM.cpp:225-238 (single level: lev 0)
  const Real dx0 = L.geom.CellSize(0);
  L.tau = Real(3.0) * Real(c.nu) / dx0 + Real(0.5);
  L.dt = dx0;

  // BCs, AmrCoreLBM.cpp:254-353
  int bc_lo[AMREX_SPACEDIM], bc_hi[AMREX_SPACEDIM];
  if (!L.geom.isAllPeriodic()) {
    for (int d = 0; d < AMREX_SPACEDIM; ++d) {
      bc_lo[d] = c.bc_lo[d];
      bc_hi[d] = c.bc_hi[d];
      L.bcval.lo_rho[d] = Real(c.bc_lo_rho[d]);
      L.bcval.lo_ux[d] = Real(c.bc_lo_ux[d]);
      L.bcval.lo_uy[d] = Real(c.bc_lo_uy[d]);
      L.bcval.lo_uz[d] = Real(c.bc_lo_uz[d]);
      L.bcval.hi_rho[d] = Real(c.bc_hi_rho[d]);
      L.bcval.hi_ux[d] = Real(c.bc_hi_ux[d]);
      L.bcval.hi_uy[d] = Real(c.bc_hi_uy[d]);
      L.bcval.hi_uz[d] = Real(c.bc_hi_uz[d]);
    }
  } else {
    for (int d = 0; d < AMREX_SPACEDIM; ++d) {
      bc_lo[d] = bc_hi[d] = BCType::int_dir;
      L.bcval.lo_rho[d] = L.bcval.lo_ux[d] = L.bcval.lo_uy[d] = L.bcval.lo_uz[d] = 0;
      L.bcval.hi_rho[d] = L.bcval.hi_ux[d] = L.bcval.hi_uy[d] = L.bcval.hi_uz[d] = 0;
    }
  }
  L.bcval.ndir = L.ndir;
  for (int q = 0; q < L.ndir; ++q) {
    L.bcval.dirx[q] = L.dirx[q];
    L.bcval.diry[q] = L.diry[q];
    L.bcval.dirz[q] = L.dirz[q];
    L.bcval.wi[q] = L.wi[q];
  }
  L.bcsMeso.assign(L.ndir, BCRec());
  L.bcsMacro.assign(L.nmac, BCRec());
  for (auto *v : {&L.bcsMeso, &L.bcsMacro})
    for (auto &r : *v)
      for (int d = 0; d < AMREX_SPACEDIM; ++d) {
        r.setLo(d, bc_lo[d]);
        r.setHi(d, bc_hi[d]);
      }
  std::memset(L.rec, 0, sizeof(L.rec));
}

// InitEquilibrium (AmrCoreLBM.cpp:2117-2164) over the whole fab box.
void init_equilibrium(RefLevel &L) {
  const Box gb = L.f_new[0].box();
  auto rho = L.macro_new[0].const_array(0);
  auto ux = L.macro_new[0].const_array(1);
  auto uy = L.macro_new[0].const_array(2);
  auto uz = L.macro_new[0].const_array(3);
  auto f = L.f_new[0].array();
  auto fo = L.f_old[0].array();
  const Real *wi = L.wi.data(), *cx = L.dirx.data(), *cy = L.diry.data(), *cz = L.dirz.data();
  const int nd = L.ndir;
  for_box(gb, [&](int i, int j, int k) {
    Real r = amrex::max(rho(i, j, k), Real(1.e-12));
    Real u0 = ux(i, j, k), v0 = uy(i, j, k), w0 = uz(i, j, k);
    Real u2 = u0 * u0 + v0 * v0 + w0 * w0;
    for (int q = 0; q < nd; ++q) {
      Real cu = cx[q] * u0 + cy[q] * v0 + cz[q] * w0;
      Real feq = wi[q] * r * (Real(1.0) + Real(3.0) * cu + Real(4.5) * cu * cu - Real(1.5) * u2);
      f(i, j, k, q) = feq;
      fo(i, j, k, q) = feq;
    }
  });
  MultiFab::Copy(L.macro_old, L.macro_new, 0, 0, L.nmac, L.nghost);
}

// AmrCoreLBM::ComputeIBForce, Source/Core/AmrCoreLBM.cpp:456-631 (no file output).
void compute_ib_force(RefLevel &L) {
  if (!L.use_ib) return;
  const Real dt_lev = L.dt;
  Real Fs[3] = {0, 0, 0};
  {
    auto F = L.forcing[0].const_array();
    const Box dom = L.geom.Domain();
    for (int n = 0; n < 3; ++n) {
      Real s = 0;
      MultiFab::forBox(dom, [&](const IntVect &iv) { s += F(iv, n); });
      Fs[n] = s;
    }
  }
#if (AMREX_SPACEDIM != 3)
  Fs[2] = 0.0;
#endif
  const auto dx = L.geom.CellSizeArray();
  Real dV = dx[0];
  dV *= dx[1];
#if (AMREX_SPACEDIM == 3)
  dV *= dx[2];
#endif
  Real Feul[3], Fm[3] = {0, 0, 0}, Fme[3], Fb[3], Ftc[3];
  for (int n = 0; n < 3; ++n) Feul[n] = -(Fs[n] * dV) / dt_lev;
  if (L.ibm) {
    auto s = L.ibm->last_marker_force_sum();
    for (int n = 0; n < 3; ++n) Fm[n] = -s[n];
  }
  for (int n = 0; n < 3; ++n) Fme[n] = Feul[n];
  for (int n = 0; n < 3; ++n) {
    Fb[n] = Feul[n];
    if (L.ibc.force_eval_method == 2) Fb[n] = Fm[n];
    else if (L.ibc.force_eval_method == 0) Fb[n] = Fme[n];
  }
  for (int n = 0; n < 3; ++n) {
    Ftc[n] = Fb[n];
    if (L.have_prev) Ftc[n] = Real(0.5) * (L.prev_body[n] + Fb[n]);
    L.prev_body[n] = Fb[n];
  }
  L.have_prev = true;
  const Real rho_ref = 1.0, U_ref = Real(L.ibc.U0), D_ref = Real(2.0) * Real(L.ibc.R);
#if (AMREX_SPACEDIM == 3)
  const Real A_ref = Math::pi<Real>() * Real(L.ibc.R) * Real(L.ibc.R);
  const Real denom = Real(0.5) * rho_ref * U_ref * U_ref * A_ref;
#else
  const Real denom = Real(0.5) * rho_ref * U_ref * U_ref * D_ref;
#endif
  double *r = L.rec;
  for (int n = 0; n < 3; ++n) {
    r[0 + n] = Ftc[n];
    r[6 + n] = Fb[n];
    r[9 + n] = Feul[n];
    r[12 + n] = Fm[n];
    r[15 + n] = Fme[n];
  }
  r[3] = r[4] = r[5] = 0;
  if (denom > 0) {
    r[3] = Ftc[0] / denom;
    r[4] = Ftc[1] / denom;
#if (AMREX_SPACEDIM == 3)
    r[5] = Ftc[2] / denom;
#endif
  }
}

// One level step: AdvancePhiAtLevel (Source/Core/AdvanceLBMAtLevel.cpp:20-394)
// for the finest (and only) level.
void advance(RefLevel &L) {
  std::swap(L.f_new, L.f_old);          // :23
  std::swap(L.macro_new, L.macro_old);  // :24
  const int ng = L.nghost;
  const Box vbx = L.ba[0];

  MultiFab &fx_cc = L.fx_cc, &fy_cc = L.fy_cc, &fz_cc = L.fz_cc;  // :43-48
  fx_cc.setVal(0.0);
  fy_cc.setVal(0.0);
  fz_cc.setVal(0.0);
  if (L.c.use_prescribed_force) {  // :52-56
    fx_cc.setVal(Real(L.c.prescribed_force[0]));
    fy_cc.setVal(Real(L.c.prescribed_force[1]));
    fz_cc.setVal(Real(L.c.prescribed_force[2]));
  }
  MultiFab &sfS = L.sfS, &smS = L.smS;  // :57-60
  fill_patch(L, sfS, L.f_old, L.ndir, L.bcsMeso, mesoscopicBcFill{L.bcval});
  fill_patch(L, smS, L.macro_old, L.nmac, L.bcsMacro, macroBcFill{L.bcval});

  if (L.use_ib && L.ibm) {  // :73-93
    MultiFab rhocc(L.ba, L.dm, 1, ng), ucc(L.ba, L.dm, 1, ng), vcc(L.ba, L.dm, 1, ng);
    MultiFab::Copy(rhocc, smS, 0, 0, 1, ng);
    MultiFab::Copy(ucc, smS, 1, 0, 1, ng);
    MultiFab::Copy(vcc, smS, 2, 0, 1, ng);
#if (AMREX_SPACEDIM == 3)
    MultiFab wcc(L.ba, L.dm, 1, ng);
    MultiFab::Copy(wcc, smS, 3, 0, 1, ng);
#else
    MultiFab wcc(L.ba, L.dm, 1, 0);
    wcc.setVal(0.0);
#endif
    MultiFab pFx(L.ba, L.dm, 1, ng), pFy(L.ba, L.dm, 1, ng), pFz(L.ba, L.dm, 1, ng);
    MultiFab::Copy(pFx, L.forcing, 0, 0, 1, ng);
    MultiFab::Copy(pFy, L.forcing, 1, 0, 1, ng);
    MultiFab::Copy(pFz, L.forcing, 2, 0, 1, ng);
    L.ibm->update_forcing(rhocc, ucc, vcc, wcc, fx_cc, fy_cc, fz_cc, L.dt, L.time, &pFx,
                          &pFy, &pFz);
  }

  if (L.use_ib) {  // pack forcing[lev] on valid cells, :122-153
    auto Fx = L.forcing[0].array(0);
    auto Fy = L.forcing[0].array(1);
    auto Fz = L.forcing[0].array(2);
    auto fx = fx_cc[0].const_array();
    auto fy = fy_cc[0].const_array();
    auto fz = fz_cc[0].const_array();
    for_box(vbx, [&](int i, int j, int k) {
      Fx(i, j, k) = fx(i, j, k, 0);
      Fy(i, j, k) = fy(i, j, k, 0);
      Fz(i, j, k) = fz(i, j, k, 0);
    });
  }
  {
    auto d = L.last_fx[0].array();
    auto fx = fx_cc[0].const_array();
    auto fy = fy_cc[0].const_array();
    auto fz = fz_cc[0].const_array();
    for_box(vbx, [&](int i, int j, int k) {
      d(i, j, k, 0) = fx(i, j, k, 0);
      d(i, j, k, 1) = fy(i, j, k, 0);
      d(i, j, k, 2) = fz(i, j, k, 0);
    });
  }

  fx_cc.FillBoundary(L.geom.periodicity());  // :192-194
  fy_cc.FillBoundary(L.geom.periodicity());
  fz_cc.FillBoundary(L.geom.periodicity());

  const Real temptau = L.tau;
  const Real *dirx_d = L.dirx.data(), *diry_d = L.diry.data(), *dirz_d = L.dirz.data();
  const Real *wi_d = L.wi.data();
  const int ndir_l = L.ndir;

  {  // collide, :207-240
    Array4<Real> rho_old = smS[0].array(0);
    Array4<Real> u_old = smS[0].array(1);
    Array4<Real> v_old = smS[0].array(2);
    Array4<Real> w_old = smS[0].array(3);
    Array4<Real> statein = sfS[0].array();
    auto fx = fx_cc[0].array(0);
    auto fy = fy_cc[0].array(0);
    auto fz = fz_cc[0].array(0);
    for_box(vbx, [&](int i, int j, int k) {
      const Real rho_loc = rho_old(i, j, k);
      const Real u_loc = u_old(i, j, k);
      const Real v_loc = v_old(i, j, k);
      const Real w_loc = w_old(i, j, k);
      Real feq_loc[BCBuf::MAX_NDIR];
      for (int q = 0; q < ndir_l; ++q)
        feq_loc[q] = feqFunction(wi_d[q], dirx_d[q], diry_d[q], dirz_d[q], rho_loc, u_loc,
                                 v_loc, w_loc);
      collide_forced(i, j, k, statein, feq_loc, ndir_l, temptau, wi_d, dirx_d, diry_d, dirz_d,
                     rho_loc, u_loc, v_loc, w_loc, fx(i, j, k), fy(i, j, k), fz(i, j, k));
    });
  }

  sfS.FillBoundary(L.geom.periodicity());  // :244

  {  // halfway bounce-back ghosts for user_1 faces, :272-373
    Array4<Real> statein = sfS[0].array();
    const Box domain = L.geom.Domain();
    const BCRec bc_rec = L.bcsMeso.empty() ? BCRec() : L.bcsMeso[0];
    Box gtbx = vbx;
    gtbx.grow(ng);
    MultiFab::forBox(gtbx, [&](const IntVect &iv) {
      const int i = iv[0], j = iv[1];
#if (AMREX_SPACEDIM == 3)
      const int k = iv[2];
#else
      const int k = 0;
#endif
      if (vbx.contains(i, j, k)) return;
      bool has_bb = false, unsupported = false;
      for (int d = 0; d < AMREX_SPACEDIM; ++d) {
        if (iv[d] < domain.smallEnd(d)) {
          if (bc_rec.lo(d) == BCType::user_1) has_bb = true;
          else unsupported = true;
        } else if (iv[d] > domain.bigEnd(d)) {
          if (bc_rec.hi(d) == BCType::user_1) has_bb = true;
          else unsupported = true;
        }
      }
      if (!has_bb || unsupported) return;
      for (int q = 0; q < ndir_l; ++q) {
        const int itgt = i + static_cast<int>(dirx_d[q]);
        const int jtgt = j + static_cast<int>(diry_d[q]);
#if (AMREX_SPACEDIM == 3)
        const int ktgt = k + static_cast<int>(dirz_d[q]);
#else
        const int ktgt = k;
#endif
        if (!vbx.contains(itgt, jtgt, ktgt)) continue;
        const int rx = -static_cast<int>(dirx_d[q]);
        const int ry = -static_cast<int>(diry_d[q]);
#if (AMREX_SPACEDIM == 3)
        const int rz = -static_cast<int>(dirz_d[q]);
#else
        const int rz = 0;
#endif
        int q_reflect = q;
        for (int p = 0; p < ndir_l; ++p) {
          if (static_cast<int>(dirx_d[p]) == rx && static_cast<int>(diry_d[p]) == ry &&
              static_cast<int>(dirz_d[p]) == rz) {
            q_reflect = p;
            break;
          }
        }
        statein(i, j, k, q) = statein(itgt, jtgt, ktgt, q_reflect);
      }
    });
  }

  {  // stream + macro, :376-386
    Array4<Real> statein = sfS[0].array();
    Array4<Real> stateout = L.f_new[0].array();
    Array4<Real> rho = L.macro_new[0].array(0);
    Array4<Real> u = L.macro_new[0].array(1);
    Array4<Real> v = L.macro_new[0].array(2);
    Array4<Real> w = L.macro_new[0].array(3);
    auto fx = fx_cc[0].array(0);
    auto fy = fy_cc[0].array(0);
    auto fz = fz_cc[0].array(0);
    for_box(vbx, [&](int i, int j, int k) {
      stream(i, j, k, stateout, statein, dirx_d, diry_d, dirz_d, ndir_l);
    });
    for_box(vbx, [&](int i, int j, int k) {
      calculateMacroForcing(i, j, k, stateout, rho, u, v, w, fx, fy, fz, ndir_l, dirx_d, diry_d,
                            dirz_d);
    });
  }
}

// valid-cell copy helpers, layout [comp][k][j][i]
void copy_out(const MultiFab &mf, int c0, int nc, double *out, const Box &vb) {
  auto a = mf[0].const_array();
  const Long n = vb.numPts();
  long idx = 0;
  MultiFab::forBox(vb, [&](const IntVect &iv) {
    for (int c = 0; c < nc; ++c) out[(Long)c * n + idx] = (double)a(iv, c0 + c);
    ++idx;
  });
}
void copy_in(MultiFab &mf, int c0, int nc, const double *in, const Box &vb) {
  auto a = mf[0].array();
  const Long n = vb.numPts();
  long idx = 0;
  MultiFab::forBox(vb, [&](const IntVect &iv) {
    for (int c = 0; c < nc; ++c) a(iv, c0 + c) = (Real)in[(Long)c * n + idx];
    ++idx;
  });
}

template <class Fn>
int guard(Fn &&fn) {
  try {
    fn();
    return 0;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "refcpu error: %s\n", e.what());
    return -1;
  }
}

}  // namespace

extern "C" {

int ref_dim(void) { return AMREX_SPACEDIM; }
int ref_real_bytes(void) { return (int)sizeof(amrex::Real); }

void *ref_create(const ilbm_case *c) {
  auto *L = new RefLevel();
  if (guard([&] { build_level(*L, *c); }) != 0) {
    delete L;
    return nullptr;
  }
  return L;
}

void ref_destroy(void *h) { delete static_cast<RefLevel *>(h); }

int ref_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

// macro fields rho,ux,uy,uz on valid cells ([4][ncell]); ghosts keep zero.
int ref_set_macro(void *h, const double *m4) {
  auto *L = static_cast<RefLevel *>(h);
  return guard([&] {
    copy_in(L->macro_new, 0, 4, m4, L->ba[0]);
    amrex::MultiFab::Copy(L->macro_old, L->macro_new, 0, 0, L->nmac, L->nghost);
  });
}
int ref_init_equilibrium(void *h) {
  auto *L = static_cast<RefLevel *>(h);
  return guard([&] { init_equilibrium(*L); });
}
int ref_set_f(void *h, const double *f) {
  auto *L = static_cast<RefLevel *>(h);
  return guard([&] { copy_in(L->f_new, 0, L->ndir, f, L->ba[0]); });
}
int ref_get_f(void *h, double *f) {
  auto *L = static_cast<RefLevel *>(h);
  return guard([&] { copy_out(L->f_new, 0, L->ndir, f, L->ba[0]); });
}
int ref_get_macro(void *h, double *m4) {
  auto *L = static_cast<RefLevel *>(h);
  return guard([&] { copy_out(L->macro_new, 0, 4, m4, L->ba[0]); });
}
// force field applied in the last step ([3][ncell]: fx_cc, fy_cc, fz_cc)
int ref_get_force(void *h, double *f3) {
  auto *L = static_cast<RefLevel *>(h);
  return guard([&] { copy_out(L->last_fx, 0, 3, f3, L->ba[0]); });
}
// set the force field of the previous step (forcing[lev], used as prev_F)
int ref_set_forcing(void *h, const double *f3) {
  auto *L = static_cast<RefLevel *>(h);
  return guard([&] { copy_in(L->forcing, 0, 3, f3, L->ba[0]); });
}

int ref_ib_create(void *h, const ilbm_ib_case *ib) {
  auto *L = static_cast<RefLevel *>(h);
  return guard([&] {
    L->ibc = *ib;
    MarkerIBParams p;
    p.coupling_method = ib->coupling_method;
    p.delta_type = ib->delta_type;
    p.loop_ns = ib->loop_ns;
    p.mdf_relax = Real(ib->mdf_relax);
    p.explicit_diag_eps = Real(ib->explicit_diag_eps);
    p.geometry_type = ib->geometry_type;
    p.box_xlo = Real(ib->box_xlo);
    p.box_xhi = Real(ib->box_xhi);
    p.box_ylo = Real(ib->box_ylo);
    p.box_yhi = Real(ib->box_yhi);
    p.box_zlo = Real(ib->box_zlo);
    p.box_zhi = Real(ib->box_zhi);
    p.box_ds = Real(ib->box_ds);
    p.box_lid_only = ib->box_lid_only;
    p.box_lid_ux = Real(ib->box_lid_ux);
    p.box_lid_uy = Real(ib->box_lid_uy);
    p.box_lid_uz = Real(ib->box_lid_uz);
    p.box_wall_tol = Real(ib->box_wall_tol);
    p.n_marker = ib->n_marker;
    p.rd = Real(ib->rd);
    p.ubx = Real(ib->ubx);
    p.uby = Real(ib->uby);
    p.ubz = Real(ib->ubz);
    p.omx = Real(ib->omx);
    p.omy = Real(ib->omy);
    p.omz = Real(ib->omz);
    p.ivc_diag_reg = Real(ib->ivc_diag_reg);
    p.ivc_rebuild_matrix = ib->ivc_rebuild_matrix;
    p.renormalize_delta = ib->renormalize_delta;
    if (p.geometry_type == MarkerIBParams::GeometryBox) {  // AmrCoreLBM.cpp:1484-1502
      const auto plo = L->geom.ProbLoArray();
      const auto phi = L->geom.ProbHiArray();
      if (p.box_xhi <= p.box_xlo) { p.box_xlo = plo[0]; p.box_xhi = phi[0]; }
      if (p.box_yhi <= p.box_ylo) { p.box_ylo = plo[1]; p.box_yhi = phi[1]; }
#if (AMREX_SPACEDIM == 3)
      if (p.box_zhi <= p.box_zlo) { p.box_zlo = plo[2]; p.box_zhi = phi[2]; }
#endif
    }
    L->ibm = std::make_unique<IBMarkerDF>(L->geom, L->dm, L->ba, Real(ib->x0), Real(ib->y0),
                                          Real(ib->z0), Real(ib->R), p);
    L->use_ib = true;
    L->forcing.setVal(0.0);
    L->have_prev = false;
  });
}

long ref_ib_num_markers(void *h) {
  auto *L = static_cast<RefLevel *>(h);
  return L->ibm ? (long)L->ibm->num_markers() : 0;
}

// marker positions and interpolated velocities at time t: [n][6] = x,y,z,u,v,w
int ref_ib_marker_state(void *h, double t, double *out6, long cap) {
  auto *L = static_cast<RefLevel *>(h);
  return guard([&] {
    std::vector<int> ids;
    std::vector<amrex::Real> data;
    L->ibm->gather_marker_state(ids, data, amrex::Real(t));
    for (size_t n = 0; n < ids.size() && (long)n < cap; ++n)
      for (int c = 0; c < 6; ++c) out6[(size_t)(ids[n] - 1) * 6 + c] = (double)data[n * 6 + c];
  });
}

int ref_ib_marker_force_sum(void *h, double *out3) {
  auto *L = static_cast<RefLevel *>(h);
  if (!L->ibm) return -1;
  auto s = L->ibm->last_marker_force_sum();
  for (int n = 0; n < 3; ++n) out3[n] = (double)s[n];
  return 0;
}

int ref_step(void *h, int nsteps) {
  auto *L = static_cast<RefLevel *>(h);
  return guard([&] {
    for (int s = 0; s < nsteps; ++s) {
      advance(*L);
      L->time += L->dt;
      ++L->step;
      compute_ib_force(*L);
    }
  });
}

double ref_time(void *h) { return (double)static_cast<RefLevel *>(h)->time; }
double ref_tau(void *h) { return (double)static_cast<RefLevel *>(h)->tau; }

int ref_force_record(void *h, double *out) {
  auto *L = static_cast<RefLevel *>(h);
  for (int n = 0; n < ILBM_FORCE_REC; ++n) out[n] = L->rec[n];
  return 0;
}

int ref_momentum_exchange(void *h, double x0, double y0, double z0, double R, int one_sided,
                          double *out3) {
  auto *L = static_cast<RefLevel *>(h);
  return guard([&] {
    LevelSetParams par;
    par.x0 = amrex::Real(x0);
    par.y0 = amrex::Real(y0);
    par.z0 = amrex::Real(z0);
    par.R = amrex::Real(R);
    auto F = IBForceEval::ComputeMomentumExchangeBodyForce(L->f_new, L->geom, L->dirx, L->diry,
                                                           L->dirz, L->ndir, par, one_sided != 0);
    for (int n = 0; n < 3; ++n) out3[n] = (double)F[n];
  });
}

// ErrorEst's field step (Source/Core/AmrCoreLBM.cpp:1020-1047): rho, u, v, w
// of macro_new FillPatched one cell out, then the reference's visPara
// (Source/LBM/visPara.H:39-54: vorticityDiagnostic and the pressure) on the
// valid cells; *vmax = vortMax.  vor / pres: valid cells, i fastest.
int ref_derived(void *h, double *vor, double *pres, double *vmax) {
  auto *L = static_cast<RefLevel *>(h);
  return guard([&] {
    MultiFab mt(L->ba, L->dm, 4, 1);
    fill_patch(*L, mt, L->macro_new, 4, L->bcsMacro, macroBcFill{L->bcval});
    MultiFab vo(L->ba, L->dm, 1, 0), pr(L->ba, L->dm, 1, 0);
    const auto dxa = L->geom.CellSizeArray();
#if (AMREX_SPACEDIM == 3)
    const Real dz = dxa[2];
#else
    const Real dz = Real(0.0);
#endif
    auto rho = mt[0].const_array(0), u = mt[0].const_array(1), v = mt[0].const_array(2),
         w = mt[0].const_array(3);
    auto va = vo[0].array(), pa = pr[0].array();
    const Box vb = L->ba[0];
    for_box(vb, [&](int i, int j, int k) {
      visPara(i, j, k, rho, u, v, w, va, pa, dxa[0], dxa[1], dz, Real(0.0));
    });
    copy_out(vo, 0, 1, vor, vb);
    copy_out(pr, 0, 1, pres, vb);
    double m = -1e300;
    MultiFab::forBox(vb, [&](const IntVect &iv) { m = std::max(m, (double)va(iv, 0)); });
    *vmax = m;
  });
}

// ErrorEst's tag loop (AmrCoreLBM.cpp:1073-1180, restated glue) around the
// reference's vorticity_tagging / levelset_tagging (Source/Tagging.H:12-35),
// with phi from the reference's LevelSetManager::build_from_cylinder
// (Source/LevelSet/LevelSet.cpp:36-74).  ls6: NULL or {x0, y0, z0, R,
// n_cells_band, dx_min}.  tags: valid cells, i fastest, 0/1.
int ref_tags(void *h, const double *vor, double threshold, int use_box, const double *box_lo,
             const double *box_hi, double nr_lo, double nr_hi, const double *ls6,
             unsigned char *tags) {
  auto *L = static_cast<RefLevel *>(h);
  return guard([&] {
    const Box vb = L->ba[0];
    MultiFab vo(L->ba, L->dm, 1, 0);
    copy_in(vo, 0, 1, vor, vb);
    LevelSetManager lsm;
    int nband = 0;
    Real dx_min = 0;
    if (ls6) {
      LevelSetParams par;
      par.x0 = Real(ls6[0]);
      par.y0 = Real(ls6[1]);
      par.z0 = Real(ls6[2]);
      par.R = Real(ls6[3]);
      nband = (int)ls6[4];
      dx_min = Real(ls6[5]);
      lsm.define_level(0, L->ba, L->dm, L->nghost);
      lsm.build_from_cylinder(0, L->geom, par);
    }
    std::vector<char> tb((size_t)vb.numPts(), 0);
    Array4<char> tg(tb.data(), vb, 1);
    auto vort = vo[0].const_array(0);
    const auto problo = L->geom.ProbLoArray();
    const auto probhi = L->geom.ProbHiArray();
    const auto dx = L->geom.CellSizeArray();
    const char tagval = 1, clearval = 0;
    for_box(vb, [&](int i, int j, int k) {
      const Real x = problo[0] + (Real(i) + Real(0.5)) * dx[0];
      if (nr_lo > 0.0 || nr_hi > 0.0) {
        if (x <= problo[0] + Real(nr_lo) || x >= probhi[0] - Real(nr_hi)) {
          tg(i, j, k) = clearval;
          return;
        }
      }
      vorticity_tagging(i, j, k, tg, vort, Real(threshold), tagval);
      if (ls6) {
        Array4<const Real> phi = lsm.phi_at(0)[0].const_array(0);
        levelset_tagging(i, j, k, tg, phi, dx_min, nband, tagval);
      }
      if (use_box) {
        const Real y = problo[1] + (Real(j) + Real(0.5)) * dx[1];
#if (AMREX_SPACEDIM == 3)
        const Real z = problo[2] + (Real(k) + Real(0.5)) * dx[2];
#else
        const Real z = Real(0.0);
#endif
        if (x >= box_lo[0] && x <= box_hi[0] && y >= box_lo[1] && y <= box_hi[1] &&
            z >= box_lo[2] && z <= box_hi[2])
          tg(i, j, k) = tagval;
      }
    });
    for (size_t n = 0; n < tb.size(); ++n) tags[n] = (unsigned char)tb[n];
  });
}

// Per-cell entry points for unit parity.
double ref_feq(double wi, double cx, double cy, double cz, double rho, double u, double v,
               double w) {
  return (double)feqFunction(amrex::Real(wi), amrex::Real(cx), amrex::Real(cy), amrex::Real(cz),
                             amrex::Real(rho), amrex::Real(u), amrex::Real(v), amrex::Real(w));
}
double ref_delta_function(double xf, double xp, double h, int type) {
  return (double)delta_function(amrex::Real(xf), amrex::Real(xp), amrex::Real(h), type);
}
double ref_overlap_1d(double xa, double xb, double h, int type, double plo, int ilo, int ihi) {
  return (double)overlap_1d(amrex::Real(xa), amrex::Real(xb), amrex::Real(h), type,
                            amrex::Real(plo), ilo, ihi);
}

}  // extern "C"
