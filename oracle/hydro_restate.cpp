// CPU restatement of CAMR's per-box hydro right-hand side (test oracle).
//
// This is the oracle the CUDA kernels are checked against.  It restates the
// reference's arithmetic operation by operation (same operands, same order,
// no FMA contraction: build with -ffp-contract=off) but organises the work
// the way the B200 kernels do: every face flux is computed once, on exactly
// the faces whose value reaches the box's fluxes and dsdt, instead of the
// reference's 17-27 whole-box passes over grow(bx,2).  Each function names
// the reference lines it follows.  oracle/_ref/libcamr_ref.so (the reference
// compiled as-is) pins this file: tests compare the two bit for bit.
#include <cmath>
#include <cstring>

#include "oracle_common.hpp"

namespace orc {
namespace {

inline double dmin(double a, double b) { return std::min(a, b); }
inline double dmax(double a, double b) { return std::max(a, b); }

// ---------------------------------------------------------------------------
// Conservative -> primitive.  Source/Hydro/Hydro_ctoprim.H:11-101.
void ctoprim(const Eos& eos, const Fab& u, const Fab& q, const Fab& qa,
             int i, int j, int k, double small_num, double eta1,
             int allow_negative_energy, long* nassert) {
  const double rho = u(i, j, k, URHO);
  if (!(rho > 0.)) return;
  const double rhoinv = 1.0 / rho;
  const double vx = u(i, j, k, UMX) * rhoinv;
  const double vy = u(i, j, k, UMY) * rhoinv;
  const double vz = u(i, j, k, UMZ) * rhoinv;
  const double kineng = 0.5 * rho * (vx * vx + vy * vy + vz * vz);
  q(i, j, k, QRHO) = rho;
  q(i, j, k, QU) = vx;
  q(i, j, k, QV) = vy;
  q(i, j, k, QW) = vz;
  for (int s = 0; s < NSPEC; ++s) q(i, j, k, QFS + s) = u(i, j, k, UFS + s) * rhoinv;
  if (!allow_negative_energy && !(u(i, j, k, UEDEN) > 0.)) ++*nassert;
  if ((u(i, j, k, UEDEN) - kineng) / u(i, j, k, UEDEN) > eta1) {
    q(i, j, k, QREINT) = (u(i, j, k, UEDEN) - kineng) * rhoinv;
  } else {
    q(i, j, k, QREINT) = u(i, j, k, UEINT) * rhoinv;
  }
  const double e = q(i, j, k, QREINT);
  if (!allow_negative_energy && !(u(i, j, k, UEINT) > 0.)) ++*nassert;
  for (int s = 0; s < NSPEC; ++s) q(i, j, k, s + QFS) = u(i, j, k, UFS + s) * rhoinv;
  const double t = eos.ey2t(e);
  const double p = eos.rey2p(rho, e);
  const double gam1 = eos.gamma;
  const double dpde = (eos.gamma - 1.0) * rho;
  const double dpdr_e = (eos.gamma - 1.0) * e;
  q(i, j, k, QTEMP) = t;
  q(i, j, k, QREINT) = e * rho;
  q(i, j, k, QPRES) = p;
  q(i, j, k, QGAME) = p / (e * rho) + 1.0;
  qa(i, j, k, QDPDR) = dpdr_e;
  qa(i, j, k, QDPDE) = dpde;
  qa(i, j, k, QGAMC) = gam1;
  const double cs = std::sqrt(gam1 * p / rho);
  qa(i, j, k, QC) = cs;
  qa(i, j, k, QCSML) = dmax(small_num, small_num * cs);
}

// Source -> primitive source (CTU only).  Hydro_ctoprim.H:106-157.
void srctoprim(const Fab& q, const Fab& qa, const Fab& src, const Fab& srcq,
               int i, int j, int k) {
  const double srcrho = src(i, j, k, URHO);
  if (q(i, j, k, QRHO) > 0.) {
    const double rhoinv = 1.0 / q(i, j, k, QRHO);
    const double vx = q(i, j, k, QU), vy = q(i, j, k, QV), vz = q(i, j, k, QW);
    const double smx = src(i, j, k, UMX), smy = src(i, j, k, UMY), smz = src(i, j, k, UMZ);
    srcq(i, j, k, QRHO) = srcrho;
    srcq(i, j, k, QU) = (smx - vx * srcrho) * rhoinv;
    srcq(i, j, k, QV) = (smy - vy * srcrho) * rhoinv;
    srcq(i, j, k, QW) = (smz - vz * srcrho) * rhoinv;
    srcq(i, j, k, QREINT) = src(i, j, k, UEINT);
    for (int s = 0; s < NSPEC; ++s) {
      srcq(i, j, k, QFS + s) = (src(i, j, k, UFS + s) - q(i, j, k, QFS + s) * srcrho) * rhoinv;
    }
    srcq(i, j, k, QPRES) =
        qa(i, j, k, QDPDE) *
            (srcq(i, j, k, QREINT) - q(i, j, k, QREINT) * srcrho * rhoinv) * rhoinv +
        qa(i, j, k, QDPDR) * srcrho;
  } else {
    srcq(i, j, k, QRHO) = 0.;
    srcq(i, j, k, QU) = 0.;
    srcq(i, j, k, QV) = 0.;
    srcq(i, j, k, QW) = 0.;
    srcq(i, j, k, QPRES) = 0.;
    srcq(i, j, k, QREINT) = 0.;
  }
}

// ---------------------------------------------------------------------------
// Two-shock approximate Riemann solver.  Source/Hydro/Hydro_riemann.H:8-173.
struct RiemannOut {
  double ustar;
  double f_rho, f_un, f_ut1, f_ut2, f_eden, f_eint;
  double q_un, q_ut1, q_ut2, q_pres, q_game;
};

RiemannOut riemannus(double rl_in, double ul, double vl, double v2l, double pl_in,
                     double rel, double rr_in, double ur, double vr, double v2r,
                     double pr_in, double rer, double cav, double gamcl, double gamcr,
                     double small, double smallc, double small_dens,
                     double small_pres, double smallu) {
  RiemannOut o;
  const double wsmall = smallc * small_dens;
  const double rl = dmax(rl_in, small_dens);
  const double pl = dmax(pl_in, small_pres);
  const double rr = dmax(rr_in, small_dens);
  const double pr = dmax(pr_in, small_pres);
  const double wl = dmax(wsmall, std::sqrt(std::fabs(gamcl * pl * rl)));
  const double wr = dmax(wsmall, std::sqrt(std::fabs(gamcr * pr * rr)));
  double pstar = ((wr * pl + wl * pr) + wl * wr * (ul - ur)) / (wl + wr);
  pstar = dmax(pstar, small_pres);
  double ustar = ((wl * ul + wr * ur) + (pl - pr)) / (wl + wr);
  bool mask = std::fabs(ustar) < smallu * 0.5 * (std::fabs(ul) + std::fabs(ur));
  ustar = mask ? 0.0 : ustar;

  double ro, uo, po, reo, gamco;
  if (ustar > 0.) {
    ro = rl; uo = ul; po = pl; reo = rel; gamco = gamcl;
  } else if (ustar < 0) {
    ro = rr; uo = ur; po = pr; reo = rer; gamco = gamcr;
  } else {
    ro = 0.5 * (rl + rr);
    uo = 0.5 * (ul + ur);
    po = 0.5 * (pl + pr);
    reo = 0.5 * (rel + rer);
    gamco = 0.5 * (gamcl + gamcr);
  }
  ro = dmax(ro, small_dens);
  const double roinv = 1.0 / ro;
  double co = std::sqrt(std::fabs(gamco * po * roinv));
  co = dmax(smallc, co);
  const double co2inv = 1.0 / (co * co);
  const double drho = (pstar - po) * co2inv;
  double rstar = ro + drho;
  rstar = dmax(small_dens, rstar);
  const double entho = (reo + po) * roinv * co2inv;
  const double estar = reo + (pstar - po) * entho;
  double cstar = std::sqrt(std::fabs(gamco * pstar / rstar));
  cstar = dmax(cstar, smallc);
  const double sgnm = (ustar < 0.) ? -1.0 : 1.0;
  double spout = co - sgnm * uo;
  double spin = cstar - sgnm * ustar;
  const double ushock = 0.5 * (spin + spout);
  if (pstar - po > 0.0) {
    spin = ushock;
    spout = ushock;
  }
  double scr;
  if (spout - spin == 0.0) {
    scr = small * cav;
  } else {
    scr = spout - spin;
  }
  double frac = (1.0 + (spout + spin) / scr) * 0.5;
  frac = dmax(0.0, dmin(1.0, frac));

  mask = ustar > 0.0;
  double qint_iv1 = mask ? vl : vr;
  double qint_iv2 = mask ? v2l : v2r;
  mask = (ustar == 0.0);
  qint_iv1 = mask ? 0.5 * (vl + vr) : qint_iv1;
  qint_iv2 = mask ? 0.5 * (v2l + v2r) : qint_iv2;

  double rho_gd = frac * rstar + (1.0 - frac) * ro;
  double qint_iu = frac * ustar + (1.0 - frac) * uo;
  double qint_gdpres = frac * pstar + (1.0 - frac) * po;
  double re_gd = frac * estar + (1.0 - frac) * reo;
  mask = (spout < 0.0);
  rho_gd = mask ? ro : rho_gd;
  qint_iu = mask ? uo : qint_iu;
  qint_gdpres = mask ? po : qint_gdpres;
  re_gd = mask ? reo : re_gd;
  mask = (spin >= 0.0);
  rho_gd = mask ? rstar : rho_gd;
  qint_iu = mask ? ustar : qint_iu;
  qint_gdpres = mask ? pstar : qint_gdpres;
  re_gd = mask ? estar : re_gd;

  const double qint_gdgame = qint_gdpres / re_gd + 1.0;
  qint_gdpres = dmax(qint_gdpres, small_pres);

  o.ustar = ustar;
  o.f_rho = rho_gd * qint_iu;
  o.f_un = o.f_rho * qint_iu + qint_gdpres;
  o.f_ut1 = o.f_rho * qint_iv1;
  o.f_ut2 = o.f_rho * qint_iv2;
  const double rhoetot =
      re_gd + 0.5 * rho_gd * (qint_iu * qint_iu + qint_iv1 * qint_iv1 + qint_iv2 * qint_iv2);
  o.f_eden = qint_iu * (rhoetot + qint_gdpres);
  o.f_eint = qint_iu * re_gd;
  o.q_un = qint_iu;
  o.q_ut1 = qint_iv1;
  o.q_ut2 = qint_iv2;
  o.q_pres = qint_gdpres;
  o.q_game = qint_gdgame;
  return o;
}

// HLLC (riemann_solver = 1), an option the reference does not have: Toro,
// "Riemann Solvers and Numerical Methods for Fluid Dynamics", 3rd ed.,
// sec. 10.4-10.6, with Davis wave speeds; rho e is carried like a passive
// density.  Interface values: the normal velocity and pressure of the
// region holding x/t = 0.  The operation order is the one the device
// kernels use, so both round alike.
RiemannOut hllc(double rl_in, double ul, double vl, double v2l, double pl_in, double rel,
                double rr_in, double ur, double vr, double v2r, double pr_in, double rer,
                double gamcl, double gamcr, double smallc, double small_dens,
                double small_pres) {
  RiemannOut o;
  const double rl = dmax(rl_in, small_dens);
  const double pl = dmax(pl_in, small_pres);
  const double rr = dmax(rr_in, small_dens);
  const double pr = dmax(pr_in, small_pres);
  const double cl = dmax(smallc, std::sqrt(std::fabs(gamcl * pl / rl)));
  const double cr = dmax(smallc, std::sqrt(std::fabs(gamcr * pr / rr)));
  const double sl = dmin(ul - cl, ur - cr);
  const double sr = dmax(ul + cl, ur + cr);
  const double el = rel + 0.5 * rl * (ul * ul + vl * vl + v2l * v2l);
  const double er = rer + 0.5 * rr * (ur * ur + vr * vr + v2r * v2r);
  const double dl = rl * (sl - ul);
  const double dr = rr * (sr - ur);
  const double sstar = ((pr - pl) + (ul * dl - ur * dr)) / (dl - dr);
  const double pstar = pl + dl * (sstar - ul);
  const bool left = sstar >= 0.0;
  const double rk = left ? rl : rr, uk = left ? ul : ur, vk = left ? vl : vr;
  const double v2k = left ? v2l : v2r, pk = left ? pl : pr, ek = left ? el : er;
  const double rek = left ? rel : rer, sk = left ? sl : sr;
  double f_rho = rk * uk;
  double f_un = rk * uk * uk + pk;
  double f_ut1 = rk * uk * vk;
  double f_ut2 = rk * uk * v2k;
  double f_eden = uk * (ek + pk);
  double f_eint = uk * rek;
  double q_un = uk, q_pres = pk;
  const bool star = left ? (sl < 0.0) : (sr > 0.0);
  if (star) {
    const double fac = rk * (sk - uk) / (sk - sstar);
    const double fac_e = rek * (sk - uk) / (sk - sstar);
    const double estar = fac * (ek / rk + (sstar - uk) * (sstar + pk / (rk * (sk - uk))));
    f_rho = f_rho + sk * (fac - rk);
    f_un = f_un + sk * (fac * sstar - rk * uk);
    f_ut1 = f_ut1 + sk * (fac * vk - rk * vk);
    f_ut2 = f_ut2 + sk * (fac * v2k - rk * v2k);
    f_eden = f_eden + sk * (estar - ek);
    f_eint = f_eint + sk * (fac_e - rek);
    q_un = sstar;
    q_pres = pstar;
  }
  o.ustar = q_un;
  o.f_rho = f_rho;
  o.f_un = f_un;
  o.f_ut1 = f_ut1;
  o.f_ut2 = f_ut2;
  o.f_eden = f_eden;
  o.f_eint = f_eint;
  o.q_un = q_un;
  o.q_ut1 = (q_un > 0.0) ? vl : (q_un < 0.0) ? vr : 0.5 * (vl + vr);
  o.q_ut2 = (q_un > 0.0) ? v2l : (q_un < 0.0) ? v2r : 0.5 * (v2l + v2r);
  o.q_pres = dmax(q_pres, small_pres);
  o.q_game = 0.5 * (gamcl + gamcr);
  return o;
}

// Component maps of one direction (Hydro_cmpflx.H:181-223).
struct DirMap {
  int iu, iv, iv2;  // primitive velocity slots (normal, transverse 1, 2)
  int gu, gv, gv2;  // Riemann-output velocity slots
  int fu, fv, fv2;  // conserved momentum slots
};
inline DirMap dirmap(int dir) {
  if (dir == 0) return {QU, QV, QW, GDU, GDV, GDW, UMX, UMY, UMZ};
  if (dir == 1) return {QV, QU, QW, GDV, GDU, GDW, UMY, UMX, UMZ};
  return {QW, QU, QV, GDW, GDU, GDV, UMZ, UMX, UMY};
}

// Face flux from left/right states.  Source/Hydro/Hydro_cmpflx.H:153-311.
// ql/qr are QVAR-long and modified in place at a physical boundary face
// exactly as the reference modifies its state arrays (:239-282).
// qaL/qaR are the qaux records of the cells left/right of the face.
void cmpflx(double* ql, double* qr, const double* qaL, const double* qaR,
            int dir, int idx, int bclo, int bchi, int domlo, int domhi,
            const orc_params& p, double* flx /*NVAR*/, double* qint /*NGDNV*/) {
  const DirMap m = dirmap(dir);
  const double cav = 0.5 * (qaR[QC] + qaL[QC]);
  const double smallc = dmax(qaR[QCSML], qaL[QCSML]);
  double gamcl = qaL[QGAMC];
  double gamcr = qaR[QGAMC];
  double ul = ql[m.iu], vl = ql[m.iv], v2l = ql[m.iv2];
  double ur = qr[m.iu], vr = qr[m.iv], v2r = qr[m.iv2];
  if (idx == domlo) {
    if (bclo == ORC_SYMMETRY || bclo == ORC_SLIPWALL || bclo == ORC_NOSLIPWALL) {
      ql[QRHO] = qr[QRHO];
      ql[QPRES] = qr[QPRES];
      ql[QREINT] = qr[QREINT];
      gamcl = gamcr;
      ul = -ur;
      vl = vr;
      v2l = v2r;
    } else if (bclo == ORC_OUTFLOW) {
      ul = ur;
      vl = vr;
      v2l = v2r;
      gamcl = gamcr;
      ql[QRHO] = qr[QRHO];
      ql[QPRES] = qr[QPRES];
      ql[QREINT] = qr[QREINT];
    }
  }
  if (idx == domhi + 1) {
    if (bchi == ORC_SYMMETRY || bchi == ORC_SLIPWALL || bchi == ORC_NOSLIPWALL) {
      qr[QRHO] = ql[QRHO];
      qr[QPRES] = ql[QPRES];
      qr[QREINT] = ql[QREINT];
      gamcr = gamcl;
      ur = -ul;
      vr = vl;
      v2r = v2l;
    } else if (bchi == ORC_OUTFLOW) {
      qr[QRHO] = ql[QRHO];
      qr[QPRES] = ql[QPRES];
      qr[QREINT] = ql[QREINT];
      gamcr = gamcl;
      ur = ul;
      vr = vl;
      v2r = v2l;
    }
  }
  const RiemannOut o =
      (p.riemann_solver == 1)
          ? hllc(ql[QRHO], ul, vl, v2l, ql[QPRES], ql[QREINT], qr[QRHO], ur, vr, v2r,
                 qr[QPRES], qr[QREINT], gamcl, gamcr, smallc, p.small_dens, p.small_pres)
          : riemannus(ql[QRHO], ul, vl, v2l, ql[QPRES], ql[QREINT], qr[QRHO], ur, vr, v2r,
                      qr[QPRES], qr[QREINT], cav, gamcl, gamcr, p.small, smallc, p.small_dens,
                      p.small_pres, p.smallu);
  flx[URHO] = o.f_rho;
  flx[m.fu] = o.f_un;
  flx[m.fv] = o.f_ut1;
  flx[m.fv2] = o.f_ut2;
  flx[UEDEN] = o.f_eden;
  flx[UEINT] = o.f_eint;
  qint[m.gu] = o.q_un;
  qint[m.gv] = o.q_ut1;
  qint[m.gv2] = o.q_ut2;
  qint[GDPRES] = o.q_pres;
  qint[GDGAME] = o.q_game;
  const double flxrho = flx[URHO];
  for (int s = 0; s < NSPEC; ++s) {
    const int n = UFS + s, nq = QFS + s;
    if (o.ustar > 0.0) {
      flx[n] = flxrho * ql[nq];
    } else if (o.ustar < 0.0) {
      flx[n] = flxrho * qr[nq];
    } else {
      flx[n] = flxrho * 0.50 * (ql[nq] + qr[nq]);
    }
  }
}

// ---------------------------------------------------------------------------
// Shock flattening.  Source/Hydro/Godunov/flatten.H:19-99.  The caller's q
// covers every cell it asks about plus the +-3 stencil, so the reference's
// "stencil leaves the q box" early return never fires for those cells.
double flatten(const Fab& q, int i, int j, int k, int dir) {
  const int e[3] = {dir == 0, dir == 1, dir == 2};
  auto Q = [&](int s, int n) { return q(i + s * e[0], j + s * e[1], k + s * e[2], n); };
  if (!q.contains(i + 3 * e[0], j + 3 * e[1], k + 3 * e[2]) ||
      !q.contains(i - 3 * e[0], j - 3 * e[1], k - 3 * e[2])) {
    return 1.0;
  }
  const int n = QPRES;
  const double small_pres = 1.e-200;
  const double shktst = 0.33e0;
  const double zcut1 = 0.75e0;
  const double zcut2 = 0.85e0;
  const double dzcut = 1.0 / (zcut2 - zcut1);
  const double qm = Q(-1, n);
  const double qp = Q(1, n);
  const double qmun = Q(-1, QU + dir);
  const double qpun = Q(1, QU + dir);
  const double qmm = Q(-2, n);
  const double qpp = Q(2, n);
  double dp = qp - qm;
  const int ishft = (dp > 0.0) ? 1 : -1;
  double denom = dmax(small_pres, std::fabs(qpp - qmm));
  double zeta = std::fabs(dp) / denom;
  const double z = dmin(1.0, dmax(0.0, dzcut * (zeta - zcut1)));
  double tst = (qmun - qpun >= 0.0) ? 1.0 : 0.0;
  double tmp = dmin(qp, qm);
  const double chi = (std::fabs(dp) / tmp) > shktst ? tst : 0.0;
  const double qpshft = Q(1 - ishft, n);
  const double qmshft = Q(-(1 + ishft), n);
  const double qpunshft = Q(1 - ishft, QU + dir);
  const double qmunshft = Q(-(1 + ishft), QU + dir);
  const double qppshft = Q(2 - ishft, n);
  const double qmmshft = Q(-(2 + ishft), n);
  dp = qpshft - qmshft;
  denom = dmax(small_pres, std::fabs(qppshft - qmmshft));
  zeta = std::fabs(dp) / denom;
  const double z2 = dmin(1.0, dmax(0.0, dzcut * (zeta - zcut1)));
  tst = (qmunshft - qpunshft >= 0.0) ? 1.0 : 0.0;
  tmp = dmin(qpshft, qmshft);
  const double chi2 = (std::fabs(dp) / tmp) > shktst ? tst : 0.0;
  return 1.0 - dmax(chi2 * z2, chi * z);
}

// ---------------------------------------------------------------------------
// PPM reconstruction and wave integrals.  Source/Hydro/Godunov/PPM.H:25-183.
void ppm_reconstruct(const double* s, double flatn, double& sm, double& sp) {
  double dsl = 2.0 * (s[1] - s[0]);
  double dsr = 2.0 * (s[2] - s[1]);
  double dsvl_l = 0.0;
  if (dsl * dsr > 0.0) {
    const double dsc = 0.5 * (s[2] - s[0]);
    dsvl_l = std::copysign(1.0, dsc) * dmin(std::fabs(dsc), dmin(std::fabs(dsl), std::fabs(dsr)));
  }
  dsl = 2.0 * (s[2] - s[1]);
  dsr = 2.0 * (s[3] - s[2]);
  double dsvl_r = 0.0;
  if (dsl * dsr > 0.0) {
    const double dsc = 0.5 * (s[3] - s[1]);
    dsvl_r = std::copysign(1.0, dsc) * dmin(std::fabs(dsc), dmin(std::fabs(dsl), std::fabs(dsr)));
  }
  sm = 0.5 * (s[2] + s[1]) - (1.0 / 6.0) * (dsvl_r - dsvl_l);
  sm = dmax(sm, dmin(s[2], s[1]));
  sm = dmin(sm, dmax(s[2], s[1]));

  dsl = 2.0 * (s[2] - s[1]);
  dsr = 2.0 * (s[3] - s[2]);
  dsvl_l = 0.0;
  if (dsl * dsr > 0.0) {
    const double dsc = 0.5 * (s[3] - s[1]);
    dsvl_l = std::copysign(1.0, dsc) * dmin(std::fabs(dsc), dmin(std::fabs(dsl), std::fabs(dsr)));
  }
  dsl = 2.0 * (s[3] - s[2]);
  dsr = 2.0 * (s[4] - s[3]);
  dsvl_r = 0.0;
  if (dsl * dsr > 0.0) {
    const double dsc = 0.5 * (s[4] - s[2]);
    dsvl_r = std::copysign(1.0, dsc) * dmin(std::fabs(dsc), dmin(std::fabs(dsl), std::fabs(dsr)));
  }
  sp = 0.5 * (s[3] + s[2]) - (1.0 / 6.0) * (dsvl_r - dsvl_l);
  sp = dmax(sp, dmin(s[3], s[2]));
  sp = dmin(sp, dmax(s[3], s[2]));

  sm = flatn * sm + (1.0 - flatn) * s[2];
  sp = flatn * sp + (1.0 - flatn) * s[2];

  if ((sp - s[2]) * (s[2] - sm) <= 0.0) {
    sp = s[2];
    sm = s[2];
  } else if (std::fabs(sp - s[2]) >= 2.0 * std::fabs(sm - s[2])) {
    sp = 3.0 * s[2] - 2.0 * sm;
  } else if (std::fabs(sm - s[2]) >= 2.0 * std::fabs(sp - s[2])) {
    sm = 3.0 * s[2] - 2.0 * sp;
  }
}

void ppm_int_profile(double sm, double sp, double sc, double u, double c,
                     double dtdx, double* Ip, double* Im) {
  const double s6 = 6.0 * sc - 3.0 * (sm + sp);
  const double speeds[3] = {u - c, u, u + c};
  for (int w = 0; w < 3; ++w) {
    const double speed = speeds[w];
    const double sigma = std::fabs(speed) * dtdx;
    if (speed <= 0.0) {
      Ip[w] = sp;
      Im[w] = sm + 0.5 * sigma * (sp - sm + (1.0 - (2.0 / 3.0) * sigma) * s6);
    } else {
      Ip[w] = sp - 0.5 * sigma * (sp - sm - (1.0 - (2.0 / 3.0) * sigma) * s6);
      Im[w] = sm;
    }
  }
}

// Normal-predictor states of one cell in direction idir by PPM with
// characteristic tracing.  Source/Hydro/Godunov/PPM.cpp:101-410.
// qp_out: the "plus" state on the cell's low face; qm_out: the "minus" state
// on its high face (QVAR slots; QGAME/QTEMP are not produced, as in the
// reference, whose consumers never read them).
void trace_ppm_cell(const Fab& q, const Fab& qa, int i, int j, int k, int idir,
                    double flat, double dt, const double dx[3],
                    const orc_params& p, double* qp_out, double* qm_out) {
  const double dtdx = dt / dx[idir];
  int QUN, QUT, QUTT;
  if (idir == 0) { QUN = QU; QUT = QV; QUTT = QW; }
  else if (idir == 1) { QUN = QV; QUT = QW; QUTT = QU; }
  else { QUN = QW; QUT = QU; QUTT = QV; }
  const int e[3] = {idir == 0, idir == 1, idir == 2};
  auto at = [&](const Fab& f, int s, int n) {
    return f(i + s * e[0], j + s * e[1], k + s * e[2], n);
  };
  const double cc = std::sqrt(qa(i, j, k, QGAMC) * q(i, j, k, QPRES) / q(i, j, k, QRHO));
  const double un = q(i, j, k, QUN);

  double Ip[QVAR + 1][3];
  double Im[QVAR + 1][3];
  for (int n = 0; n < QVAR; ++n) {
    if (n == QGAME || n == QTEMP) continue;  // traced by the reference, never read
    double s[5];
    for (int o = 0; o < 5; ++o) s[o] = at(q, o - 2, n);
    double sm, sp;
    ppm_reconstruct(s, flat, sm, sp);
    ppm_int_profile(sm, sp, s[2], un, cc, dtdx, Ip[n], Im[n]);
  }
  {
    double s[5];
    for (int o = 0; o < 5; ++o) s[o] = at(qa, o - 2, QGAMC);
    double sm, sp;
    ppm_reconstruct(s, flat, sm, sp);
    ppm_int_profile(sm, sp, s[2], un, cc, dtdx, Ip[QVAR], Im[QVAR]);
  }
  for (int s = 0; s < NSPEC; ++s) {
    qp_out[QFS + s] = Im[QFS + s][1];
    qm_out[QFS + s] = Ip[QFS + s][1];
  }
  // plus state on face i (PPM.cpp:204-310)
  {
    double rho_ref = Im[QRHO][0];
    const double un_ref = Im[QUN][0];
    double p_ref = Im[QPRES][0];
    const double rhoe_g_ref = Im[QREINT][0];
    const double gam_ref = Im[QVAR][0];
    rho_ref = dmax(rho_ref, p.small_dens);
    const double rho_ref_inv = 1.0 / rho_ref;
    p_ref = dmax(p_ref, p.small_pres);
    const double cc_ref = std::sqrt(gam_ref * p_ref / rho_ref);
    const double csq_ref = cc_ref * cc_ref;
    const double cc_ref_inv = 1.0 / cc_ref;
    const double h_g_ref = (p_ref + rhoe_g_ref) * rho_ref_inv / csq_ref;
    const double dum = un_ref - Im[QUN][0];
    const double dptotm = p_ref - Im[QPRES][0];
    const double drho = rho_ref - Im[QRHO][1];
    const double dptot = p_ref - Im[QPRES][1];
    const double drhoe_g = rhoe_g_ref - Im[QREINT][1];
    const double dup = un_ref - Im[QUN][2];
    const double dptotp = p_ref - Im[QPRES][2];
    double alpham = 0.5 * (dptotm * rho_ref_inv * cc_ref_inv - dum) * rho_ref * cc_ref_inv;
    double alphap = 0.5 * (dptotp * rho_ref_inv * cc_ref_inv + dup) * rho_ref * cc_ref_inv;
    double alpha0r = drho - dptot / csq_ref;
    double alpha0e_g = drhoe_g - dptot * h_g_ref;
    if (un - cc > 0.) alpham = 0.;
    else if (un - cc < 0.) alpham *= -1.0;
    else alpham *= -0.5;
    if (un + cc > 0.) alphap = 0.;
    else if (un + cc < 0.) alphap *= -1.0;
    else alphap *= -0.5;
    if (un > 0.) { alpha0r = 0.; alpha0e_g = 0.; }
    else if (un < 0.) { alpha0r *= -1.0; alpha0e_g *= -1.0; }
    else { alpha0r *= -0.5; alpha0e_g *= -0.5; }
    qp_out[QRHO] = rho_ref + alphap + alpham + alpha0r;
    qp_out[QUN] = un_ref + (alphap - alpham) * cc_ref * rho_ref_inv;
    qp_out[QPRES] = p_ref + (alphap + alpham) * csq_ref;
    qp_out[QRHO] = dmax(qp_out[QRHO], p.small_dens);
    qp_out[QPRES] = dmax(qp_out[QPRES], p.small_pres);
    qp_out[QUT] = Im[QUT][1];
    qp_out[QUTT] = Im[QUTT][1];
    qp_out[QREINT] = rhoe_g_ref + (alphap + alpham) * h_g_ref * csq_ref + alpha0e_g;
  }
  // minus state on face i+1 (PPM.cpp:313-409)
  {
    double rho_ref = Ip[QRHO][2];
    const double un_ref = Ip[QUN][2];
    double p_ref = Ip[QPRES][2];
    const double rhoe_g_ref = Ip[QREINT][2];
    const double gam_ref = Ip[QVAR][2];
    rho_ref = dmax(rho_ref, p.small_dens);
    const double rho_ref_inv = 1.0 / rho_ref;
    p_ref = dmax(p_ref, p.small_pres);
    const double cc_ref = std::sqrt(gam_ref * p_ref / rho_ref);
    const double csq_ref = cc_ref * cc_ref;
    const double cc_ref_inv = 1.0 / cc_ref;
    const double h_g_ref = (p_ref + rhoe_g_ref) * rho_ref_inv / csq_ref;
    const double dum = un_ref - Ip[QUN][0];
    const double dptotm = p_ref - Ip[QPRES][0];
    const double drho = rho_ref - Ip[QRHO][1];
    const double dptot = p_ref - Ip[QPRES][1];
    const double drhoe_g = rhoe_g_ref - Ip[QREINT][1];
    const double dup = un_ref - Ip[QUN][2];
    const double dptotp = p_ref - Ip[QPRES][2];
    double alpham = 0.5 * (dptotm * rho_ref_inv * cc_ref_inv - dum) * rho_ref * cc_ref_inv;
    double alphap = 0.5 * (dptotp * rho_ref_inv * cc_ref_inv + dup) * rho_ref * cc_ref_inv;
    double alpha0r = drho - dptot / csq_ref;
    double alpha0e_g = drhoe_g - dptot * h_g_ref;
    if (un - cc > 0.) alpham *= -1.0;
    else if (un - cc < 0.) alpham = 0.;
    else alpham *= -0.5;
    if (un + cc > 0.) alphap *= -1.0;
    else if (un + cc < 0.) alphap = 0.;
    else alphap *= -0.5;
    if (un > 0.) { alpha0r *= -1.0; alpha0e_g *= -1.0; }
    else if (un < 0.) { alpha0r = 0.; alpha0e_g = 0.; }
    else { alpha0r *= -0.5; alpha0e_g *= -0.5; }
    qm_out[QRHO] = rho_ref + alphap + alpham + alpha0r;
    qm_out[QUN] = un_ref + (alphap - alpham) * cc_ref * rho_ref_inv;
    qm_out[QPRES] = p_ref + (alphap + alpham) * csq_ref;
    qm_out[QRHO] = dmax(qm_out[QRHO], p.small_dens);
    // The reference floors this pressure with small_dens (PPM.cpp:398).
    qm_out[QPRES] = dmax(qm_out[QPRES], p.small_dens);
    qm_out[QUT] = Ip[QUT][1];
    qm_out[QUTT] = Ip[QUTT][1];
    qm_out[QREINT] = rhoe_g_ref + (alphap + alpham) * h_g_ref * csq_ref + alpha0e_g;
  }
}

// ---------------------------------------------------------------------------
// PLM slopes and characteristic tracing.  Source/Hydro/Godunov/PLM.H:19-323.
double plm_slope(const Fab& q, int i, int j, int k, int n, int dir, double flat, int order) {
  if (order == 1) return 0.;
  const int e[3] = {dir == 0, dir == 1, dir == 2};
  auto Q = [&](int s) { return q(i + s * e[0], j + s * e[1], k + s * e[2], n); };
  double dlft, drgt, dcen, dfm = 0.0, dfp = 0.0, dlim, dsgn, dtemp;
  const double qc = Q(0), qm2 = Q(-2), qm = Q(-1), qp = Q(1), qp2 = Q(2);
  if (order == 4) {
    dlft = qm - qm2;
    drgt = qc - qm;
    dcen = 0.5 * (dlft + drgt);
    dsgn = std::copysign(1.0, dcen);
    dlim = (dlft * drgt >= 0.0) ? 2.0 * dmin(std::fabs(dlft), std::fabs(drgt)) : 0.0;
    dfm = dsgn * dmin(dlim, std::fabs(dcen));
    dlft = qp - qc;
    drgt = qp2 - qp;
    dcen = 0.5 * (dlft + drgt);
    dsgn = std::copysign(1.0, dcen);
    dlim = (dlft * drgt >= 0.0) ? 2.0 * dmin(std::fabs(dlft), std::fabs(drgt)) : 0.0;
    dfp = dsgn * dmin(dlim, std::fabs(dcen));
  }
  dlft = qc - qm;
  drgt = qp - qc;
  dcen = 0.5 * (dlft + drgt);
  dsgn = std::copysign(1.0, dcen);
  dlim = (dlft * drgt >= 0.0) ? 2.0 * dmin(std::fabs(dlft), std::fabs(drgt)) : 0.0;
  dtemp = 4.0 / 3.0 * dcen - 1.0 / 6.0 * (dfp + dfm);
  return flat * dsgn * dmin(dlim, std::fabs(dtemp));
}

double plm_pslope(const Fab& q, const Fab& srcQ, int i, int j, int k, int n, int dir,
                  double dx, double flat, int order) {
  if (order == 1) return 0.;
  const int e[3] = {dir == 0, dir == 1, dir == 2};
  auto Q = [&](int s, int c) { return q(i + s * e[0], j + s * e[1], k + s * e[2], c); };
  auto S = [&](int s, int c) { return srcQ(i + s * e[0], j + s * e[1], k + s * e[2], c); };
  const int QIU = QU + dir;
  double dlft, drgt, dcen, dfm = 0.0, dfp = 0.0, dlim, dsgn, dtemp;
  const double qc = Q(0, n), qm2 = Q(-2, n), qm = Q(-1, n), qp = Q(1, n), qp2 = Q(2, n);
  if (order == 4) {
    dlft = qm - qm2 - 0.25 * dx * (Q(-1, QRHO) + Q(-2, QRHO)) * (S(-1, QIU) + S(-2, QIU));
    drgt = qc - qm - 0.25 * dx * (Q(-1, QRHO) + Q(0, QRHO)) * (S(-1, QIU) + S(0, QIU));
    dcen = 0.5 * (dlft + drgt);
    dsgn = std::copysign(1.0, dcen);
    dlim = (dlft * drgt >= 0.0) ? 2.0 * dmin(std::fabs(dlft), std::fabs(drgt)) : 0.0;
    dfm = dsgn * dmin(dlim, std::fabs(dcen));
    dlft = qp - qc - 0.25 * dx * (Q(1, QRHO) + Q(0, QRHO)) * (S(1, QIU) + S(0, QIU));
    drgt = qp2 - qp - 0.25 * dx * (Q(1, QRHO) + Q(2, QRHO)) * (S(1, QIU) + S(2, QIU));
    dcen = 0.5 * (dlft + drgt);
    dsgn = std::copysign(1.0, dcen);
    dlim = (dlft * drgt >= 0.0) ? 2.0 * dmin(std::fabs(dlft), std::fabs(drgt)) : 0.0;
    dfp = dsgn * dmin(dlim, std::fabs(dcen));
  }
  dlft = qc - qm - 0.25 * dx * (Q(0, QRHO) + Q(-1, QRHO)) * (S(0, QIU) + S(-1, QIU));
  drgt = qp - qc - 0.25 * dx * (Q(0, QRHO) + Q(1, QRHO)) * (S(0, QIU) + S(1, QIU));
  dcen = 0.5 * (dlft + drgt);
  dsgn = std::copysign(1.0, dcen);
  dlim = (dlft * drgt >= 0.0) ? 2.0 * dmin(std::fabs(dlft), std::fabs(drgt)) : 0.0;
  dtemp = 4.0 / 3.0 * dcen - 1.0 / 6.0 * (dfp + dfm);
  double dp = flat * dsgn * dmin(dlim, std::fabs(dtemp));
  dp += Q(0, QRHO) * S(0, QIU) * dx;
  return dp;
}

// hydro_plm_d (PLM.H:170-323): qp_out on the low face, qm_out on the high face.
void trace_plm_cell(const Fab& q, double cc, const double* slope, int i, int j, int k,
                    int dir, double dx, double dt, const orc_params& p,
                    double* qp_out, double* qm_out) {
  const int l0 = dir;
  const int l1 = (dir == 0) ? 1 : 0;
  const int l2 = (dir == 2) ? 1 : 2;
  const double dtdx = dt / dx;
  const double cs = cc * cc;
  const double rho = q(i, j, k, QRHO);
  const double vel[3] = {q(i, j, k, QU), q(i, j, k, QV), q(i, j, k, QW)};
  const double pr = q(i, j, k, QPRES);
  const double rhoe = q(i, j, k, QREINT);
  const double enth = ((rhoe + pr) / rho) / cs;
  const double drho = slope[QRHO];
  const double dvel[3] = {slope[QU], slope[QV], slope[QW]};
  const double dp = slope[QPRES];
  const double drhoe = slope[QREINT];
  const double alpham = 0.5 * (dp / (rho * cc) - dvel[dir]) * rho / cc;
  const double alphap = 0.5 * (dp / (rho * cc) + dvel[dir]) * rho / cc;
  const double alpha0r = drho - dp / cs;
  const double alpha0e = drhoe - dp * enth;
  const double alpha0v = dvel[l1];
  const double alpha0w = dvel[l2];
  const double wv[3] = {vel[dir] - cc, vel[dir], vel[dir] + cc};
  {
    const double rho_ref = rho - 0.5 * (1.0 + dtdx * dmin(wv[0], 0.0)) * drho;
    double vel_ref[3];
    for (int d = 0; d < 3; ++d)
      vel_ref[d] = vel[d] - 0.5 * (1.0 + dtdx * dmin(wv[0], 0.0)) * dvel[d];
    const double p_ref = pr - 0.5 * (1.0 + dtdx * dmin(wv[0], 0.0)) * dp;
    const double rhoe_ref = rhoe - 0.5 * (1.0 + dtdx * dmin(wv[0], 0.0)) * drhoe;
    const double apright = 0.25 * dtdx * (wv[0] - wv[2]) * (1.0 - std::copysign(1.0, wv[2])) * alphap;
    const double amright = 0.0;
    const double azrright = 0.25 * dtdx * (wv[0] - wv[1]) * (1.0 - std::copysign(1.0, wv[1])) * alpha0r;
    const double azeright = 0.25 * dtdx * (wv[0] - wv[1]) * (1.0 - std::copysign(1.0, wv[1])) * alpha0e;
    const double azv1rght = 0.25 * dtdx * (wv[0] - wv[1]) * (1.0 - std::copysign(1.0, wv[1])) * alpha0v;
    const double azw1rght = 0.25 * dtdx * (wv[0] - wv[1]) * (1.0 - std::copysign(1.0, wv[1])) * alpha0w;
    qp_out[QRHO] = rho_ref + apright + amright + azrright;
    qp_out[QRHO] = dmax(qp_out[QRHO], p.small_dens);
    qp_out[QU + l0] = vel_ref[l0] + (apright - amright) * cc / rho;
    qp_out[QU + l1] = vel_ref[l1] + azv1rght;
    qp_out[QU + l2] = vel_ref[l2] + azw1rght;
    qp_out[QPRES] = p_ref + (apright + amright) * cs;
    qp_out[QPRES] = dmax(qp_out[QPRES], p.small_pres);
    qp_out[QREINT] = rhoe_ref + (apright + amright) * enth * cs + azeright;
  }
  {
    const double rho_ref = rho + 0.5 * (1.0 - dtdx * dmax(wv[2], 0.0)) * drho;
    double vel_ref[3];
    for (int d = 0; d < 3; ++d)
      vel_ref[d] = vel[d] + 0.5 * (1.0 - dtdx * dmax(wv[2], 0.0)) * dvel[d];
    const double p_ref = pr + 0.5 * (1.0 - dtdx * dmax(wv[2], 0.0)) * dp;
    const double rhoe_ref = rhoe + 0.5 * (1.0 - dtdx * dmax(wv[2], 0.0)) * drhoe;
    const double apleft = 0.0;
    const double amleft = 0.25 * dtdx * (wv[2] - wv[0]) * (1.0 + std::copysign(1.0, wv[0])) * alpham;
    const double azrleft = 0.25 * dtdx * (wv[2] - wv[1]) * (1.0 + std::copysign(1.0, wv[1])) * alpha0r;
    const double azeleft = 0.25 * dtdx * (wv[2] - wv[1]) * (1.0 + std::copysign(1.0, wv[1])) * alpha0e;
    const double azv1left = 0.25 * dtdx * (wv[2] - wv[1]) * (1.0 + std::copysign(1.0, wv[1])) * alpha0v;
    const double azw1left = 0.25 * dtdx * (wv[2] - wv[1]) * (1.0 + std::copysign(1.0, wv[1])) * alpha0w;
    qm_out[QRHO] = rho_ref + apleft + amleft + azrleft;
    qm_out[QRHO] = dmax(qm_out[QRHO], p.small_dens);
    qm_out[QU + l0] = vel_ref[l0] + (apleft - amleft) * cc / rho;
    qm_out[QU + l1] = vel_ref[l1] + azv1left;
    qm_out[QU + l2] = vel_ref[l2] + azw1left;
    qm_out[QPRES] = p_ref + (apleft + amleft) * cs;
    qm_out[QPRES] = dmax(qm_out[QPRES], p.small_pres);
    qm_out[QREINT] = rhoe_ref + (apleft + amleft) * enth * cs + azeleft;
  }
  for (int s = 0; s < NSPEC; ++s) {
    const int n = QFS + s;
    const double vel_ad = q(i, j, k, QU + l0);
    {
      const double spzero = (vel_ad > 0) ? -1.0 : vel_ad * dtdx;
      const double acmprght = 0.5 * (-1.0 - spzero) * slope[n];
      qp_out[n] = q(i, j, k, n) + acmprght;
    }
    {
      const double spzero = vel_ad >= 0 ? vel_ad * dtdx : 1.0;
      const double acmpleft = 0.5 * (1.0 - spzero) * slope[n];
      qm_out[n] = q(i, j, k, n) + acmpleft;
    }
  }
}

// ---------------------------------------------------------------------------
// Transverse corrections.  Source/Hydro/Godunov/Godunov_utils_3D.H.
// The reference's hydro_transdo / hydro_transdd each produce the plus state
// on a cell's low face (qp) and the minus state on its high face (qm); the two
// halves share only the cell's flux differences, so they are restated as two
// functions.  `fd` holds the cell's scaled flux differences in the order
// rho, mx, my, mz, E, species; pav/dAu/dAup the interface-pressure terms.
struct TransTerms {
  double flxrho, flxu, flxv, flxw, flxe;
  double compn[NSPEC];
  double dAup, pav, dAu;
  double c;  // qaux QGAMC of the cell
};

// hydro_transdo, :74-122 (the shared part).
TransTerms transdo_terms(const double* fl_lo, const double* fl_hi, const double* qi_lo,
                         const double* qi_hi, int qvidx, double gamc, double cdtdx) {
  TransTerms t;
  t.flxrho = cdtdx * (fl_hi[URHO] - fl_lo[URHO]);
  t.flxu = cdtdx * (fl_hi[UMX] - fl_lo[UMX]);
  t.flxv = cdtdx * (fl_hi[UMY] - fl_lo[UMY]);
  t.flxw = cdtdx * (fl_hi[UMZ] - fl_lo[UMZ]);
  t.flxe = cdtdx * (fl_hi[UEDEN] - fl_lo[UEDEN]);
  t.c = gamc;
  for (int s = 0; s < NSPEC; ++s) t.compn[s] = cdtdx * (fl_hi[UFS + s] - fl_lo[UFS + s]);
  const double pggp = qi_hi[GDPRES];
  const double pggm = qi_lo[GDPRES];
  const double ugp = qi_hi[qvidx];
  const double ugm = qi_lo[qvidx];
  t.dAup = pggp * ugp - pggm * ugm;
  t.pav = 0.5 * (pggp + pggm);
  t.dAu = ugp - ugm;
  return t;
}

// One side of hydro_transdo (:82-238): qn is the normal-predictor state on
// the face, out the corrected state (QRHO, QU..QW, QREINT, QPRES, species).
void transdo_side(const TransTerms& t, const double* qn, double cdtdx,
                  const orc_params& p, double* out) {
  for (int s = 0; s < NSPEC; ++s) {
    const int nqp = QFS + s;
    const double rr = qn[QRHO];
    const double rrnew = rr - t.flxrho;
    const double compo = rr * qn[nqp] - t.compn[s];
    out[nqp] = compo / rrnew;
  }
  const double rrr = qn[QRHO];
  double rur = qn[QU];
  double rvr = qn[QV];
  double rwr = qn[QW];
  const double ekinr = 0.5 * rrr * (rur * rur + rvr * rvr + rwr * rwr);
  rur *= rrr;
  rvr *= rrr;
  rwr *= rrr;
  const double rer = qn[QREINT] + ekinr;
  double rrnewr = rrr - t.flxrho;
  double runewr = rur - t.flxu;
  double rvnewr = rvr - t.flxv;
  double rwnewr = rwr - t.flxw;
  double renewr = rer - t.flxe;
  bool reset_state = false;
  if (p.transverse_reset_density == 1 && rrnewr < 0.) {
    rrnewr = rrr;
    runewr = rur;
    rvnewr = rvr;
    rwnewr = rwr;
    renewr = rer;
    reset_state = true;
  }
  out[QRHO] = rrnewr;
  out[QU] = runewr / rrnewr;
  out[QV] = rvnewr / rrnewr;
  out[QW] = rwnewr / rrnewr;
  const double rhoekinr = 0.5 * (runewr * runewr + rvnewr * rvnewr + rwnewr * rwnewr) / rrnewr;
  out[QREINT] = renewr - rhoekinr;
  if (!reset_state) {
    const double pnewr = qn[QPRES] - cdtdx * (t.dAup + t.pav * t.dAu * (t.c - 1.0));
    out[QPRES] = dmax(pnewr, p.small_pres);
  } else {
    out[QPRES] = qn[QPRES];
  }
}

struct TransDDTerms {
  double flxrho, flxu, flxv, flxw, flxe;
  double compn[NSPEC];
  double pxnew, pynew;
  double c;
};

// hydro_transdd, :307-384 (the shared part).
TransDDTerms transdd_terms(const double* f0_lo, const double* f0_hi, const double* f1_lo,
                           const double* f1_hi, const double* q0_lo, const double* q0_hi,
                           const double* q1_lo, const double* q1_hi, int qvidx0,
                           int qvidx1, double gamc, double cdtdx0, double cdtdx1) {
  TransDDTerms t;
  auto diff = [&](int n) {
    return cdtdx0 * (f0_hi[n] - f0_lo[n]) + cdtdx1 * (f1_hi[n] - f1_lo[n]);
  };
  t.flxrho = diff(URHO);
  t.flxu = diff(UMX);
  t.flxv = diff(UMY);
  t.flxw = diff(UMZ);
  t.flxe = diff(UEDEN);
  t.c = gamc;
  for (int s = 0; s < NSPEC; ++s) t.compn[s] = diff(UFS + s);
  const double pggpx = q0_hi[GDPRES];
  const double pggmx = q0_lo[GDPRES];
  const double ugpx = q0_hi[qvidx0];
  const double ugmx = q0_lo[qvidx0];
  const double dAupx = pggpx * ugpx - pggmx * ugmx;
  const double pavx = 0.5 * (pggpx + pggmx);
  const double dAux = ugpx - ugmx;
  const double pggpy = q1_hi[GDPRES];
  const double pggmy = q1_lo[GDPRES];
  const double ugpy = q1_hi[qvidx1];
  const double ugmy = q1_lo[qvidx1];
  const double dAupy = pggpy * ugpy - pggmy * ugmy;
  const double pavy = 0.5 * (pggpy + pggmy);
  const double dAuy = ugpy - ugmy;
  t.pxnew = cdtdx0 * (dAupx + pavx * dAux * (t.c - 1.0));
  t.pynew = cdtdx1 * (dAupy + pavy * dAuy * (t.c - 1.0));
  return t;
}

// One side of hydro_transdd (:326-481); srcq is the cell's primitive source.
void transdd_side(const TransDDTerms& t, const double* qn, const double* srcq,
                  double hdt, const orc_params& p, double* out) {
  const double rrr = qn[QRHO];
  double rrnewr = rrr - t.flxrho;
  for (int s = 0; s < NSPEC; ++s) {
    const int nqp = QFS + s;
    const double compo = rrr * qn[nqp] - t.compn[s];
    out[nqp] = compo / rrnewr + hdt * srcq[nqp];
  }
  const double rur = rrr * qn[QU];
  const double rvr = rrr * qn[QV];
  const double rwr = rrr * qn[QW];
  const double ekinr = 0.5 * (rur * rur + rvr * rvr + rwr * rwr) / rrr;
  const double rer = qn[QREINT] + ekinr;
  double runewr = rur - t.flxu;
  double rvnewr = rvr - t.flxv;
  double rwnewr = rwr - t.flxw;
  double renewr = rer - t.flxe;
  bool reset_state = false;
  if (p.transverse_reset_density == 1 && rrnewr < 0.) {
    rrnewr = rrr;
    runewr = rur;
    rvnewr = rvr;
    rwnewr = rwr;
    renewr = rer;
    reset_state = true;
  }
  out[QRHO] = rrnewr + hdt * srcq[QRHO];
  out[QU] = runewr / rrnewr + hdt * srcq[QU];
  out[QV] = rvnewr / rrnewr + hdt * srcq[QV];
  out[QW] = rwnewr / rrnewr + hdt * srcq[QW];
  const double rhoekinr = 0.5 * (runewr * runewr + rvnewr * rvnewr + rwnewr * rwnewr) / rrnewr;
  out[QREINT] = renewr - rhoekinr + hdt * srcq[QREINT];
  if (!reset_state) {
    out[QPRES] = qn[QPRES] - t.pxnew - t.pynew + hdt * srcq[QPRES];
  } else {
    out[QPRES] = qn[QPRES] + hdt * srcq[QPRES];
  }
  out[QPRES] = dmax(out[QPRES], p.small_pres);
}

// ---------------------------------------------------------------------------
// MOL characteristic slopes.  Source/Hydro/MOL/MOL_hydro_K.H:11-255.
inline double limiter(double dlft, double drgt, double plm_theta) {
  const double dcen = 0.5 * (dlft + drgt);
  const double dsgn = std::copysign(1.0, dcen);
  const double slop = plm_theta * dmin(std::fabs(dlft), std::fabs(drgt));
  const double dlim = (dlft * drgt >= 0.0) ? slop : 0.0;
  return dsgn * dmin(dlim, std::fabs(dcen));
}

// Slots written: 0 (u-c), 2 (u+c), 3, 4 (transverse velocities), QREINT,
// QFS..; slot 1 (entropy) is computed by the y/z reference versions but never
// read by mol_riemann_{x,y,z}, so it is not produced here.
void mol_slope(const Fab& q, const Fab& qa, int i, int j, int k, int dir,
               int plm_iorder, double small_dens, double* dq) {
  for (int n = 0; n < QVAR; ++n) dq[n] = 0.;
  if (plm_iorder == 1) return;
  const double plm_theta = 2.0;
  const int e[3] = {dir == 0, dir == 1, dir == 2};
  auto Q = [&](int s, int n) { return q(i + s * e[0], j + s * e[1], k + s * e[2], n); };
  const int un = QU + dir;
  const int t1 = (dir == 0) ? QV : QU;
  const int t2 = (dir == 2) ? QV : QW;
  const double c = qa(i, j, k, QC);
  double dlft = 0.5 * (Q(0, QPRES) - Q(-1, QPRES)) / c - 0.5 * Q(0, QRHO) * (Q(0, un) - Q(-1, un));
  double drgt = 0.5 * (Q(1, QPRES) - Q(0, QPRES)) / c - 0.5 * Q(0, QRHO) * (Q(1, un) - Q(0, un));
  dq[0] = limiter(dlft, drgt, plm_theta);
  const double cs2 = c * c;
  dlft = 0.5 * (Q(0, QPRES) - Q(-1, QPRES)) / c + 0.5 * Q(0, QRHO) * (Q(0, un) - Q(-1, un));
  drgt = 0.5 * (Q(1, QPRES) - Q(0, QPRES)) / c + 0.5 * Q(0, QRHO) * (Q(1, un) - Q(0, un));
  dq[2] = limiter(dlft, drgt, plm_theta);
  dlft = Q(0, t1) - Q(-1, t1);
  drgt = Q(1, t1) - Q(0, t1);
  dq[3] = limiter(dlft, drgt, plm_theta);
  dlft = Q(0, t2) - Q(-1, t2);
  drgt = Q(1, t2) - Q(0, t2);
  dq[4] = limiter(dlft, drgt, plm_theta);
  const double enth = (Q(0, QREINT) + Q(0, QPRES)) / dmax(Q(0, QRHO), small_dens);
  dlft = (Q(0, QREINT) - Q(-1, QREINT)) - enth * (Q(0, QPRES) - Q(-1, QPRES)) / cs2;
  drgt = (Q(1, QREINT) - Q(0, QREINT)) - enth * (Q(1, QPRES) - Q(0, QPRES)) / cs2;
  dq[QREINT] = limiter(dlft, drgt, plm_theta);
  for (int s = 0; s < NSPEC; ++s) {
    const int n = QFS + s;
    dlft = Q(0, QRHO) * Q(0, n) - Q(-1, QRHO) * Q(-1, n) - Q(0, n) * (Q(0, QPRES) - Q(-1, QPRES)) / cs2;
    drgt = Q(1, QRHO) * Q(1, n) - Q(0, QRHO) * Q(0, n) - Q(0, n) * (Q(1, QPRES) - Q(0, QPRES)) / cs2;
    dq[n] = limiter(dlft, drgt, plm_theta);
  }
}

// Edge states of mol_riemann_{x,y,z} (MOL_riemann_K.H:32-163, 190-320, 349-484).
// L: cell left of face f (f - e_dir), R: cell f.  qR_fallback is cell f's
// species, which the reference also uses for the LEFT state when the traced
// partial densities sum below small_dens (MOL_riemann_K.H:82-86).
void mol_edge_states(const Fab& q, const Fab& qa, const double* dqL, const double* dqR,
                     int iL, int jL, int kL, int iR, int jR, int kR, int dir,
                     double small_dens, double small_pres, double* ql, double* qr) {
  const int un = QU + dir;
  const int t1 = (dir == 0) ? QV : QU;
  const int t2 = (dir == 2) ? QV : QW;
  {
    const double cspeed = qa(iL, jL, kL, QC);
    const double enth = (q(iL, jL, kL, QREINT) + q(iL, jL, kL, QPRES)) / dmax(q(iL, jL, kL, QRHO), small_dens);
    double pl = q(iL, jL, kL, QPRES) + 0.5 * (dqL[0] + dqL[2]) * cspeed;
    pl = dmax(pl, small_pres);
    ql[QPRES] = pl;
    ql[un] = q(iL, jL, kL, un) + 0.5 * ((dqL[2] - dqL[0]) / q(iL, jL, kL, QRHO));
    ql[t1] = q(iL, jL, kL, t1) + 0.5 * dqL[3];
    ql[t2] = q(iL, jL, kL, t2) + 0.5 * dqL[4];
    double sum = 0.;
    for (int s = 0; s < NSPEC; ++s) {
      const int n = QFS + s;
      const double specden = q(iL, jL, kL, QRHO) * q(iL, jL, kL, n) +
                             0.5 * (dqL[n] + q(iL, jL, kL, n) * (dqL[0] + dqL[2]) / cspeed);
      sum += specden;
      ql[n] = specden;
    }
    if (sum < small_dens) {
      for (int s = 0; s < NSPEC; ++s) ql[QFS + s] = q(iR, jR, kR, QFS + s);
    } else {
      for (int s = 0; s < NSPEC; ++s) ql[QFS + s] = ql[QFS + s] / sum;
    }
    ql[QRHO] = dmax(sum, small_dens);
    ql[QREINT] = q(iL, jL, kL, QREINT) + 0.5 * (dqL[QREINT] + enth * (dqL[0] + dqL[2]) / cspeed);
  }
  {
    const double cspeed = qa(iR, jR, kR, QC);
    const double enth = (q(iR, jR, kR, QREINT) + q(iR, jR, kR, QPRES)) / dmax(q(iR, jR, kR, QRHO), small_dens);
    double pr = q(iR, jR, kR, QPRES) - 0.5 * (dqR[0] + dqR[2]) * cspeed;
    pr = dmax(pr, small_pres);
    qr[QPRES] = pr;
    qr[un] = q(iR, jR, kR, un) - 0.5 * ((dqR[2] - dqR[0]) / q(iR, jR, kR, QRHO));
    qr[t1] = q(iR, jR, kR, t1) - 0.5 * dqR[3];
    qr[t2] = q(iR, jR, kR, t2) - 0.5 * dqR[4];
    double sum = 0.;
    for (int s = 0; s < NSPEC; ++s) {
      const int n = QFS + s;
      const double specden = q(iR, jR, kR, QRHO) * q(iR, jR, kR, n) -
                             0.5 * (dqR[n] + q(iR, jR, kR, n) * (dqR[0] + dqR[2]) / cspeed);
      sum += specden;
      qr[n] = specden;
    }
    if (sum < small_dens) {
      for (int s = 0; s < NSPEC; ++s) qr[QFS + s] = q(iR, jR, kR, QFS + s);
    } else {
      for (int s = 0; s < NSPEC; ++s) qr[QFS + s] = qr[QFS + s] / sum;
    }
    qr[QRHO] = dmax(sum, small_dens);
    qr[QREINT] = q(iR, jR, kR, QREINT) - 0.5 * (dqR[QREINT] + enth * (dqR[0] + dqR[2]) / cspeed);
  }
}

// ---------------------------------------------------------------------------
// Nodal velocity divergence.  Source/Hydro/Hydro_utils_K.H:12-169 (3-D).
double divu_node(const Fab& q, int i, int j, int k, const double dx[3],
                 const int domlo[3], const int domhi[3], const int bclo[3],
                 const int bchi[3]) {
  const int NS = ORC_NOSLIPWALL;
  const double dxx = dx[0], dy = dx[1], dz = dx[2];
  double ux = 0.25 * (q(i, j, k, QU) - q(i - 1, j, k, QU) + q(i, j, k - 1, QU) -
                      q(i - 1, j, k - 1, QU) + q(i, j - 1, k, QU) - q(i - 1, j - 1, k, QU) +
                      q(i, j - 1, k - 1, QU) - q(i - 1, j - 1, k - 1, QU)) / dxx;
  double vy = 0.25 * (q(i, j, k, QV) - q(i, j - 1, k, QV) + q(i, j, k - 1, QV) -
                      q(i, j - 1, k - 1, QV) + q(i - 1, j, k, QV) - q(i - 1, j - 1, k, QV) +
                      q(i - 1, j, k - 1, QV) - q(i - 1, j - 1, k - 1, QV)) / dy;
  double wz = 0.25 * (q(i, j, k, QW) - q(i, j, k - 1, QW) + q(i - 1, j, k, QW) -
                      q(i - 1, j, k - 1, QW) + q(i, j - 1, k, QW) - q(i, j - 1, k - 1, QW) +
                      q(i - 1, j - 1, k, QW) - q(i - 1, j - 1, k - 1, QW)) / dz;
  if (i == domlo[0] && bclo[0] == NS) {
    vy = 0.5 * (q(i, j, k, QV) - q(i, j - 1, k, QV) + q(i, j, k - 1, QV) - q(i, j - 1, k - 1, QV)) / dy;
    wz = 0.5 * (q(i, j, k, QW) - q(i, j, k - 1, QW) + q(i, j - 1, k, QW) - q(i, j - 1, k - 1, QW)) / dz;
  } else if (i == domhi[0] + 1 && bchi[0] == NS) {
    vy = 0.5 * (q(i - 1, j, k, QV) - q(i - 1, j - 1, k, QV) + q(i - 1, j, k - 1, QV) - q(i - 1, j - 1, k - 1, QV)) / dy;
    wz = 0.5 * (q(i - 1, j, k, QW) - q(i - 1, j, k - 1, QW) + q(i - 1, j - 1, k, QW) - q(i - 1, j - 1, k - 1, QW)) / dz;
  }
  if (j == domlo[1] && bclo[1] == NS) {
    ux = 0.5 * (q(i, j, k, QU) - q(i - 1, j, k, QU) + q(i, j, k - 1, QU) - q(i - 1, j, k - 1, QU)) / dxx;
    wz = 0.5 * (q(i, j, k, QW) - q(i, j, k - 1, QW) + q(i - 1, j, k, QW) - q(i - 1, j, k - 1, QW)) / dz;
  } else if (j == domhi[1] + 1 && bchi[1] == NS) {
    ux = 0.5 * (q(i, j - 1, k, QU) - q(i - 1, j - 1, k, QU) + q(i, j - 1, k - 1, QU) - q(i - 1, j - 1, k - 1, QU)) / dxx;
    wz = 0.5 * (q(i, j - 1, k, QW) - q(i, j - 1, k - 1, QW) + q(i - 1, j - 1, k, QW) - q(i - 1, j - 1, k - 1, QW)) / dz;
  }
  if (k == domlo[2] && bclo[2] == NS) {
    ux = 0.5 * (q(i, j, k, QU) - q(i - 1, j, k, QU) + q(i, j - 1, k, QU) - q(i - 1, j - 1, k, QU)) / dxx;
    vy = 0.5 * (q(i, j, k, QV) - q(i, j - 1, k, QV) + q(i - 1, j, k, QV) - q(i - 1, j - 1, k, QV)) / dy;
  } else if (k == domhi[2] + 1 && bchi[2] == NS) {
    ux = 0.5 * (q(i, j, k - 1, QU) - q(i - 1, j, k - 1, QU) + q(i, j - 1, k - 1, QU) - q(i - 1, j - 1, k - 1, QU)) / dxx;
    vy = 0.5 * (q(i, j, k - 1, QV) - q(i, j - 1, k - 1, QV) + q(i - 1, j, k - 1, QV) - q(i - 1, j - 1, k - 1, QV)) / dy;
  }
  if (j == domlo[1] && bclo[1] == NS && k == domlo[2] && bclo[2] == NS) {
    ux = (q(i, j, k, QU) - q(i - 1, j, k, QU)) / dxx;
  } else if ((j == domhi[1] + 1 && bchi[1] == NS) && (k == domlo[2] && bclo[2] == NS)) {
    ux = (q(i, j - 1, k, QU) - q(i - 1, j - 1, k, QU)) / dxx;
  } else if ((j == domlo[1] && bclo[1] == NS) && (k == domhi[2] + 1 && bchi[2] == NS)) {
    ux = (q(i, j, k - 1, QU) - q(i - 1, j, k - 1, QU)) / dxx;
  } else if ((j == domhi[1] + 1 && bchi[1] == NS) && (k == domhi[2] + 1 && bchi[2] == NS)) {
    ux = (q(i, j - 1, k - 1, QU) - q(i - 1, j - 1, k - 1, QU)) / dxx;
  }
  if (i == domlo[0] && bclo[0] == NS && k == domlo[2] && bclo[2] == NS) {
    vy = (q(i, j, k, QV) - q(i, j - 1, k, QV)) / dy;
  } else if ((i == domhi[0] + 1 && bchi[0] == NS) && (k == domlo[2] && bclo[2] == NS)) {
    vy = (q(i - 1, j, k, QV) - q(i - 1, j - 1, k, QV)) / dy;
  } else if ((i == domlo[0] && bclo[0] == NS) && (k == domhi[2] + 1 && bchi[2] == NS)) {
    vy = (q(i, j, k - 1, QV) - q(i, j - 1, k - 1, QV)) / dy;
  } else if ((i == domhi[0] + 1 && bchi[0] == NS) && (k == domhi[2] + 1 && bchi[2] == NS)) {
    vy = (q(i - 1, j, k - 1, QV) - q(i - 1, j - 1, k - 1, QV)) / dy;
  }
  if (i == domlo[0] && bclo[0] == NS && j == domlo[1] && bclo[1] == NS) {
    wz = (q(i, j, k, QW) - q(i, j, k - 1, QW)) / dz;
  } else if ((i == domhi[0] + 1 && bchi[0] == NS) && (j == domlo[1] && bclo[1] == NS)) {
    wz = (q(i - 1, j, k, QW) - q(i - 1, j, k - 1, QW)) / dz;
  } else if ((i == domlo[0] && bclo[0] == NS) && (j == domhi[1] + 1 && bchi[1] == NS)) {
    wz = (q(i, j - 1, k, QW) - q(i, j - 1, k - 1, QW)) / dz;
  } else if ((i == domhi[0] + 1 && bchi[0] == NS) && (j == domhi[1] + 1 && bchi[1] == NS)) {
    wz = (q(i - 1, j - 1, k, QW) - q(i - 1, j - 1, k - 1, QW)) / dz;
  }
  return ux + vy + wz;
}

// adjust_fluxes at one face (Hydro_adjust_fluxes.cpp:13-44): artificial
// viscosity (hydro_artif_visc.H:7-64), species normalisation
// (Hydro_utils_K.H:207-219), area weighting (:224-234).
void adjust_flux(double* flx, const Fab& divu, const Fab& u, int i, int j, int k,
                 int dir, double dx, double difmag, int domlo, int domhi, int bclo,
                 int bchi, double area) {
  const int e[3] = {dir == 0, dir == 1, dir == 2};
  const int t1 = (dir == 0) ? 1 : 0;
  const int t2 = (dir == 2) ? 1 : 2;
  const int a1[3] = {t1 == 0, t1 == 1, t1 == 2};
  const int a2[3] = {t2 == 0, t2 == 1, t2 == 2};
  const double div =
      difmag * dmin(0.0, 0.25 * (divu(i, j, k) + divu(i + a1[0], j + a1[1], k + a1[2]) +
                                 divu(i + a2[0], j + a2[1], k + a2[2]) +
                                 divu(i + a1[0] + a2[0], j + a1[1] + a2[1], k + a1[2] + a2[2])));
  const int idx = (dir == 0) ? i : (dir == 1) ? j : k;
  const bool at_bndry = (idx == domlo && bclo == ORC_NOSLIPWALL) ||
                        (idx == domhi + 1 && bchi == ORC_NOSLIPWALL);
  for (int n = 0; n < NVAR; ++n) {
    if (n == UTEMP) continue;
    const bool is_tang_vel = (dir == 0 && (n == UMY || n == UMZ)) ||
                             (dir == 1 && (n == UMX || n == UMZ)) ||
                             (dir == 2 && (n == UMX || n == UMY));
    if (!(at_bndry && is_tang_vel)) {
      flx[n] += dx * div * (u(i, j, k, n) - u(i - e[0], j - e[1], k - e[2], n));
    }
  }
  flx[UTEMP] = 0.0;
  double summ = 0.0;
  for (int n = UFS; n < UFS + NSPEC; ++n) summ += flx[n];
  const double fac = (summ != 0.0) ? flx[URHO] / summ : 1.0;
  for (int n = UFS; n < UFS + NSPEC; ++n) flx[n] *= fac;
  for (int n = 0; n < NVAR; ++n) flx[n] *= area;
}

}  // namespace

// ---------------------------------------------------------------------------
// One box.  Mirrors construct_hydro_source's per-box body + hydro_umdrv.
long hydro_box_restated(const orc_params& p, const Box3& bx, const int dom_lo[3],
                        const int dom_hi[3], const int bclo[3], const int bchi[3],
                        const Fab& u, const Fab* src, const Fab& dsdt, Fab flx[3],
                        const double dx[3], double dt) {
  long nassert = 0;
  const Eos eos{p.eos_gamma};
  const Box3 g4 = grow(bx, 4);
  const Box3 g1 = grow(bx, 1);
  Fab q(g4.lo, g4.hi, QVAR), qa(g4.lo, g4.hi, NQAUX);
  for_box(g4, [&](int i, int j, int k) {
    ctoprim(eos, u, q, qa, i, j, k, p.small_num, p.dual_energy_eta1,
            p.allow_negative_energy, &nassert);
  });
  const double area[3] = {dx[1] * dx[2], dx[0] * dx[2], dx[0] * dx[1]};
  const double vol = dx[0] * dx[1] * dx[2];

  // Final fluxes on the faces of bx (NVAR) and their Riemann interface values.
  Fab qint_final[3];
  for (int d = 0; d < 3; ++d) {
    const Box3 fb = faces(bx, d);
    qint_final[d].alloc(fb.lo, fb.hi, NGDNV);
    for_box(fb, [&](int i, int j, int k) {
      for (int n = 0; n < NVAR; ++n) flx[d](i, j, k, n) = 0.0;
    });
  }

  if (!p.do_mol) {
    // ---- CTU (Godunov_umeth, Source/Hydro/Godunov/Godunov_3D.cpp:12-460) ----
    Fab srcq(g4.lo, g4.hi, QVAR);
    Fab zero;
    const Fab* sp = src;
    if (!sp) {
      zero.alloc(g4.lo, g4.hi, NVAR);
      for (auto& v : zero.own) v = 0.0;
      sp = &zero;
    }
    for_box(g4, [&](int i, int j, int k) { srctoprim(q, qa, *sp, srcq, i, j, k); });

    const double hdt = 0.5 * dt;
    const double hdtd[3] = {0.5 * dt / dx[0], 0.5 * dt / dx[1], 0.5 * dt / dx[2]};
    const double cdtd[3] = {1.0 / 3.0 * dt / dx[0], 1.0 / 3.0 * dt / dx[1],
                            1.0 / 3.0 * dt / dx[2]};

    // Normal predictor on grow(bx,1): sm[d] holds the minus (left) state and
    // sp_[d] the plus (right) state, both indexed by face.
    Fab smf[3], spf[3];
    for (int d = 0; d < 3; ++d) {
      Box3 fb = faces(g1, d);
      fb.lo[d] = g1.lo[d];
      smf[d].alloc(fb.lo, fb.hi, QVAR);
      spf[d].alloc(fb.lo, fb.hi, QVAR);
    }
    for_box(g1, [&](int i, int j, int k) {
      double flat = 1.0;
      if (p.use_flattening == 1) {
        for (int df = 0; df < 3; ++df) flat = dmin(flat, flatten(q, i, j, k, df));
      }
      for (int d = 0; d < 3; ++d) {
        const int e[3] = {d == 0, d == 1, d == 2};
        double qp_o[QVAR], qm_o[QVAR];
        for (int n = 0; n < QVAR; ++n) qp_o[n] = qm_o[n] = std::numeric_limits<double>::quiet_NaN();
        if (p.ppm_type == 0) {
          double slope[QVAR];
          for (int n = 0; n < QVAR; ++n) {
            if (n == QPRES && p.use_pslope)
              slope[n] = plm_pslope(q, srcq, i, j, k, n, d, dx[d], flat, p.plm_iorder);
            else
              slope[n] = plm_slope(q, i, j, k, n, d, flat, p.plm_iorder);
          }
          trace_plm_cell(q, qa(i, j, k, QC), slope, i, j, k, d, dx[d], dt, p, qp_o, qm_o);
        } else {
          trace_ppm_cell(q, qa, i, j, k, d, flat, dt, dx, p, qp_o, qm_o);
        }
        for (int n = 0; n < QVAR; ++n) {
          spf[d](i, j, k, n) = qp_o[n];
          smf[d](i + e[0], j + e[1], k + e[2], n) = qm_o[n];
        }
      }
    });

    auto load = [](const Fab& f, int i, int j, int k, double* out) {
      for (int n = 0; n < f.nc; ++n) out[n] = f(i, j, k, n);
    };
    auto qarec = [&](int i, int j, int k, double* out) {
      for (int n = 0; n < NQAUX; ++n) out[n] = qa(i, j, k, n);
    };

    // First-pass fluxes in each direction E on E-faces [lo,hi+1] x g1.
    Fab f1[3], g1q[3];
    for (int E = 0; E < 3; ++E) {
      Box3 fb = faces(g1, E);
      fb.lo[E] = bx.lo[E];
      fb.hi[E] = bx.hi[E] + 1;
      f1[E].alloc(fb.lo, fb.hi, NVAR);
      g1q[E].alloc(fb.lo, fb.hi, NGDNV);
      const int e[3] = {E == 0, E == 1, E == 2};
      for_box(fb, [&](int i, int j, int k) {
        double ql[QVAR], qr[QVAR], aL[NQAUX], aR[NQAUX], fl[NVAR], gi[NGDNV];
        for (int n = 0; n < NVAR; ++n) fl[n] = 0.0;
        for (int n = 0; n < NGDNV; ++n) gi[n] = 0.0;
        load(smf[E], i, j, k, ql);
        load(spf[E], i, j, k, qr);
        qarec(i - e[0], j - e[1], k - e[2], aL);
        qarec(i, j, k, aR);
        const int idx = (E == 0) ? i : (E == 1) ? j : k;
        cmpflx(ql, qr, aL, aR, E, idx, bclo[E], bchi[E], dom_lo[E], dom_hi[E], p, fl, gi);
        // The reference's first-pass cmpflx edits the predictor states in
        // place at a physical boundary face; later passes read them.
        for (int n = 0; n < QVAR; ++n) {
          smf[E](i, j, k, n) = ql[n];
          spf[E](i, j, k, n) = qr[n];
        }
        for (int n = 0; n < NVAR; ++n) f1[E](i, j, k, n) = fl[n];
        for (int n = 0; n < NGDNV; ++n) g1q[E](i, j, k, n) = gi[n];
      });
    }

    // Second pass: D-faces corrected by E-fluxes (reference "D|E"), on
    // D-faces [lo,hi+1], F (third direction) in g1, E in bx.
    Fab f2[3][3], g2q[3][3];
    for (int D = 0; D < 3; ++D) {
      for (int E = 0; E < 3; ++E) {
        if (E == D) continue;
        const int F = 3 - D - E;
        Box3 fb = faces(bx, D);
        fb.lo[F] -= 1;
        fb.hi[F] += 1;
        f2[D][E].alloc(fb.lo, fb.hi, NVAR);
        g2q[D][E].alloc(fb.lo, fb.hi, NGDNV);
        const int eD[3] = {D == 0, D == 1, D == 2};
        const int eE[3] = {E == 0, E == 1, E == 2};
        const int qvidx = (E == 0) ? GDU : (E == 1) ? GDV : GDW;
        for_box(fb, [&](int i, int j, int k) {
          double qm[QVAR], qp[QVAR], qn[QVAR], aL[NQAUX], aR[NQAUX];
          for (int n = 0; n < QVAR; ++n) qm[n] = qp[n] = std::numeric_limits<double>::quiet_NaN();
          double flo[NVAR], fhi[NVAR], glo[NGDNV], ghi[NGDNV];
          // minus half of cell f - e_D
          {
            const int ci = i - eD[0], cj = j - eD[1], ck = k - eD[2];
            load(f1[E], ci, cj, ck, flo);
            load(f1[E], ci + eE[0], cj + eE[1], ck + eE[2], fhi);
            load(g1q[E], ci, cj, ck, glo);
            load(g1q[E], ci + eE[0], cj + eE[1], ck + eE[2], ghi);
            const TransTerms t = transdo_terms(flo, fhi, glo, ghi, qvidx, qa(ci, cj, ck, QGAMC), cdtd[E]);
            load(smf[D], i, j, k, qn);
            transdo_side(t, qn, cdtd[E], p, qm);
          }
          // plus half of cell f
          {
            load(f1[E], i, j, k, flo);
            load(f1[E], i + eE[0], j + eE[1], k + eE[2], fhi);
            load(g1q[E], i, j, k, glo);
            load(g1q[E], i + eE[0], j + eE[1], k + eE[2], ghi);
            const TransTerms t = transdo_terms(flo, fhi, glo, ghi, qvidx, qa(i, j, k, QGAMC), cdtd[E]);
            load(spf[D], i, j, k, qn);
            transdo_side(t, qn, cdtd[E], p, qp);
          }
          qarec(i - eD[0], j - eD[1], k - eD[2], aL);
          qarec(i, j, k, aR);
          double fl[NVAR], gi[NGDNV];
          for (int n = 0; n < NVAR; ++n) fl[n] = 0.0;
          for (int n = 0; n < NGDNV; ++n) gi[n] = 0.0;
          const int idx = (D == 0) ? i : (D == 1) ? j : k;
          cmpflx(qm, qp, aL, aR, D, idx, bclo[D], bchi[D], dom_lo[D], dom_hi[D], p, fl, gi);
          for (int n = 0; n < NVAR; ++n) f2[D][E](i, j, k, n) = fl[n];
          for (int n = 0; n < NGDNV; ++n) g2q[D][E](i, j, k, n) = gi[n];
        });
      }
    }

    // Final pass: F-faces of bx corrected by "t0|t1" and "t1|t0" fluxes.
    for (int F = 0; F < 3; ++F) {
      const int t0 = (F == 0) ? 1 : 0;
      const int t1 = (F == 2) ? 1 : 2;
      const int e0[3] = {t0 == 0, t0 == 1, t0 == 2};
      const int e1[3] = {t1 == 0, t1 == 1, t1 == 2};
      const int eF[3] = {F == 0, F == 1, F == 2};
      const int qvidx0 = (F == 0) ? GDV : GDU;
      const int qvidx1 = (F == 2) ? GDV : GDW;
      const Fab& fa = f2[t0][t1];
      const Fab& fb_ = f2[t1][t0];
      const Fab& qa0 = g2q[t0][t1];
      const Fab& qb1 = g2q[t1][t0];
      for_box(faces(bx, F), [&](int i, int j, int k) {
        double qm[QVAR], qp[QVAR], qn[QVAR], sq[QVAR], aL[NQAUX], aR[NQAUX];
        for (int n = 0; n < QVAR; ++n) qm[n] = qp[n] = std::numeric_limits<double>::quiet_NaN();
        double f0lo[NVAR], f0hi[NVAR], f1lo[NVAR], f1hi[NVAR];
        double q0lo[NGDNV], q0hi[NGDNV], q1lo[NGDNV], q1hi[NGDNV];
        auto half = [&](int ci, int cj, int ck, const Fab& st, double* out) {
          load(fa, ci, cj, ck, f0lo);
          load(fa, ci + e0[0], cj + e0[1], ck + e0[2], f0hi);
          load(fb_, ci, cj, ck, f1lo);
          load(fb_, ci + e1[0], cj + e1[1], ck + e1[2], f1hi);
          load(qa0, ci, cj, ck, q0lo);
          load(qa0, ci + e0[0], cj + e0[1], ck + e0[2], q0hi);
          load(qb1, ci, cj, ck, q1lo);
          load(qb1, ci + e1[0], cj + e1[1], ck + e1[2], q1hi);
          const TransDDTerms t = transdd_terms(f0lo, f0hi, f1lo, f1hi, q0lo, q0hi, q1lo, q1hi,
                                               qvidx0, qvidx1, qa(ci, cj, ck, QGAMC),
                                               hdtd[t0], hdtd[t1]);
          load(srcq, ci, cj, ck, sq);
          transdd_side(t, qn, sq, hdt, p, out);
        };
        load(smf[F], i, j, k, qn);
        half(i - eF[0], j - eF[1], k - eF[2], smf[F], qm);
        load(spf[F], i, j, k, qn);
        half(i, j, k, spf[F], qp);
        qarec(i - eF[0], j - eF[1], k - eF[2], aL);
        qarec(i, j, k, aR);
        double fl[NVAR], gi[NGDNV];
        for (int n = 0; n < NVAR; ++n) fl[n] = 0.0;
        for (int n = 0; n < NGDNV; ++n) gi[n] = 0.0;
        const int idx = (F == 0) ? i : (F == 1) ? j : k;
        cmpflx(qm, qp, aL, aR, F, idx, bclo[F], bchi[F], dom_lo[F], dom_hi[F], p, fl, gi);
        for (int n = 0; n < NVAR; ++n) flx[F](i, j, k, n) = fl[n];
        for (int n = 0; n < NGDNV; ++n) qint_final[F](i, j, k, n) = gi[n];
      });
    }
  } else {
    // ---- MOL (MOL_umeth, Source/Hydro/MOL/MOL_umeth.cpp:15-141) ----
    for (int d = 0; d < 3; ++d) {
      const int e[3] = {d == 0, d == 1, d == 2};
      const Box3 sb = grow(bx, d, 1);
      Fab slope(sb.lo, sb.hi, QVAR);
      for_box(sb, [&](int i, int j, int k) {
        double dq[QVAR];
        mol_slope(q, qa, i, j, k, d, p.plm_iorder, p.small_dens, dq);
        for (int n = 0; n < QVAR; ++n) slope(i, j, k, n) = dq[n];
      });
      for_box(faces(bx, d), [&](int i, int j, int k) {
        const int iL = i - e[0], jL = j - e[1], kL = k - e[2];
        double dqL[QVAR], dqR[QVAR], ql[QVAR], qr[QVAR], aL[NQAUX], aR[NQAUX];
        for (int n = 0; n < QVAR; ++n) {
          dqL[n] = slope(iL, jL, kL, n);
          dqR[n] = slope(i, j, k, n);
          ql[n] = qr[n] = std::numeric_limits<double>::quiet_NaN();
        }
        mol_edge_states(q, qa, dqL, dqR, iL, jL, kL, i, j, k, d, p.small_dens, p.small_pres, ql, qr);
        for (int n = 0; n < NQAUX; ++n) { aL[n] = qa(iL, jL, kL, n); aR[n] = qa(i, j, k, n); }
        double fl[NVAR], gi[NGDNV];
        for (int n = 0; n < NVAR; ++n) fl[n] = 0.0;
        for (int n = 0; n < NGDNV; ++n) gi[n] = 0.0;
        const int idx = (d == 0) ? i : (d == 1) ? j : k;
        cmpflx(ql, qr, aL, aR, d, idx, bclo[d], bchi[d], dom_lo[d], dom_hi[d], p, fl, gi);
        for (int n = 0; n < NVAR; ++n) flx[d](i, j, k, n) = fl[n];
        for (int n = 0; n < NGDNV; ++n) qint_final[d](i, j, k, n) = gi[n];
      });
    }
  }

  // pdivu on bx from the final interface values (Hydro_utils_K.H:175-202).
  Fab pdivu(bx.lo, bx.hi, 1);
  for_box(bx, [&](int i, int j, int k) {
    const Fab& q1 = qint_final[0];
    const Fab& q2 = qint_final[1];
    const Fab& q3 = qint_final[2];
    pdivu(i, j, k) = 0.5 *
                     ((q1(i + 1, j, k, GDPRES) + q1(i, j, k, GDPRES)) *
                          (q1(i + 1, j, k, GDU) * area[0] - q1(i, j, k, GDU) * area[0]) +
                      (q2(i, j + 1, k, GDPRES) + q2(i, j, k, GDPRES)) *
                          (q2(i, j + 1, k, GDV) * area[1] - q2(i, j, k, GDV) * area[1]) +
                      (q3(i, j, k + 1, GDPRES) + q3(i, j, k, GDPRES)) *
                          (q3(i, j, k + 1, GDW) * area[2] - q3(i, j, k, GDW) * area[2])) /
                     vol;
  });

  // Nodal divu on the nodes of bx (hydro_umdrv, Hydro_umdrv.cpp:83-85).
  Box3 nb = bx;
  for (int d = 0; d < 3; ++d) nb.hi[d] += 1;
  Fab divu(nb.lo, nb.hi, 1);
  for_box(nb, [&](int i, int j, int k) {
    divu(i, j, k) = divu_node(q, i, j, k, dx, dom_lo, dom_hi, bclo, bchi);
  });

  for (int d = 0; d < 3; ++d) {
    for_box(faces(bx, d), [&](int i, int j, int k) {
      double fl[NVAR];
      for (int n = 0; n < NVAR; ++n) fl[n] = flx[d](i, j, k, n);
      adjust_flux(fl, divu, u, i, j, k, d, dx[d], p.difmag, dom_lo[d], dom_hi[d], bclo[d],
                  bchi[d], area[d]);
      for (int n = 0; n < NVAR; ++n) flx[d](i, j, k, n) = fl[n];
    });
  }

  // hydro_consup / hydro_update (Hydro_utils_K.H:239-257).
  for_box(bx, [&](int i, int j, int k) {
    const double volinv = 1.0 / vol;
    for (int n = 0; n < NVAR; ++n) {
      dsdt(i, j, k, n) += (flx[0](i, j, k, n) - flx[0](i + 1, j, k, n) + flx[1](i, j, k, n) -
                           flx[1](i, j + 1, k, n) + flx[2](i, j, k, n) - flx[2](i, j, k + 1, n)) *
                          volinv;
    }
    dsdt(i, j, k, UEINT) -= pdivu(i, j, k);
  });
  return nassert;
}

}  // namespace orc

extern "C" long orc_hydro_box(const orc_params* p, const int bx_lo[3], const int bx_hi[3],
                              const int dom_lo[3], const int dom_hi[3], const int bclo[3],
                              const int bchi[3], const double* uin, const int uin_lo[3],
                              const int uin_hi[3], const double* src, double* dsdt,
                              const int dsdt_lo[3], const int dsdt_hi[3], double* flx0,
                              double* flx1, double* flx2, const double dx[3], double dt) {
  using namespace orc;
  Box3 bx;
  for (int d = 0; d < 3; ++d) { bx.lo[d] = bx_lo[d]; bx.hi[d] = bx_hi[d]; }
  Fab u, s, dd, f[3];
  u.view(const_cast<double*>(uin), uin_lo, uin_hi, NVAR);
  if (src) s.view(const_cast<double*>(src), uin_lo, uin_hi, NVAR);
  dd.view(dsdt, dsdt_lo, dsdt_hi, NVAR);
  double* fp[3] = {flx0, flx1, flx2};
  for (int d = 0; d < 3; ++d) {
    const Box3 fb = faces(bx, d);
    f[d].view(fp[d], fb.lo, fb.hi, NVAR);
  }
  return hydro_box_restated(*p, bx, dom_lo, dom_hi, bclo, bchi, u, src ? &s : nullptr, dd, f,
                            dx, dt);
}
