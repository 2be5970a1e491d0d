// Pointwise pieces of the discrete adjoint of the MOL (SSP-RK2, PLM slopes,
// two-shock Riemann) level step: for each forward piece, a restatement of
// its arithmetic (same operations as the forward kernels) and its
// vector-Jacobian product, written out by hand in reverse order.  Branches
// (min/max, limiter cases, Riemann wave cases) take the derivative of the
// branch the forward value took.  Host and device: the CPU test suite
// checks every VJP here against finite differences of the forward.
//
// Forward pieces and the reference lines they follow:
//   face_forward   MOL edge states (Source/Hydro/MOL/MOL_riemann_K.H:12-488),
//                  hydro_cmpflx at an interior face (Hydro_cmpflx.H:153-311),
//                  riemannus (Hydro_riemann.H:8-173), adjust_fluxes' artificial
//                  viscosity, species normalisation and area scaling
//                  (hydro_artif_visc.H:7-64, Hydro_utils_K.H:207-234)
//   slope_forward  mol_slope_{x,y,z} with the MC limiter (MOL_hydro_K.H:11-255)
//   ctoprim        hydro_ctoprim (Hydro_ctoprim.H:11-101)
//   clean          normalize_species + reset_internal_energy of computeTemp
//                  (Source/CAMR.cpp:866-908, :1141-1185;
//                  Source/Utils/CAMR_reset_internal_e.H:13-129)
#pragma once

#include <cmath>

#include "rndiv.h"

#ifdef __CUDACC__
#define CAMR_HD __host__ __device__ __forceinline__
#else
#define CAMR_HD inline
#endif

namespace camr {
namespace adj {

// Slots of a primitive record (the q array of the forward kernels).
enum { QR = 0, QU = 1, QV = 2, QW = 3, QP = 4, QRE = 5, QY = 6, QC = 9, QCS = 10, NQ = 11 };
// Slots of a slope record (slot 1, the entropy wave, is never read).
enum { S0 = 0, S2 = 1, S3 = 2, S4 = 3, SRE = 4, SY = 5, NS = 8 };
// Conserved state.
enum { RHO = 0, MX = 1, MY = 2, MZ = 3, EDEN = 4, EINT = 5, TEMP = 6, FS = 7, NV = 10 };
constexpr int NSP = 3;

struct Par {
  double gamma, small, small_dens, small_pres, smallu, small_num, difmag, eta1, eta2;
  double small_temp;
  int dual_energy_update_E_from_e;
};

CAMR_HD double hmax(double a, double b) { return (a < b) ? b : a; }  // std::max
CAMR_HD double hmin(double a, double b) { return (b < a) ? b : a; }  // std::min
CAMR_HD double sgn(double x) { return (x < 0.0) ? -1.0 : 1.0; }
// Derivative of |x|, taken as 0 at x = 0 (where the limiters' |dl|, |dr|
// sit when a field is exactly flat or exactly zero).
CAMR_HD double dabs(double x) { return (x > 0.0) ? 1.0 : ((x < 0.0) ? -1.0 : 0.0); }

// ---------------------------------------------------------------------------
// Two-shock Riemann solver with its intermediates.
struct RIn {
  double rl, ul, vl, v2l, pl, rel, rr, ur, vr, v2r, pr, rer, cav, smallc;
};
struct RTape {
  double rl, pl, rr, pr, wsmall, wls, wrs, wl, wr, den, nump, pstar0, pstar, numu, ustar0;
  double ustar, ro_sel, uo, po, reo, ro, roinv, co0, co, co2inv, drho, rstar0, rstar, entho;
  double estar, cstar0, cstar, sgnm, spout0, spin0, spout, spin, scr, ratio, frac0, frac;
  double iv1, iv2, rho_gd, iu, gdp0, gdp, re_gd, frho, rhoetot;
  bool mask0, shock, scr_zero;
  int sel;   // 1: left state, -1: right state, 0: average (ustar == 0)
  int wave;  // 2: star (spin >= 0), 1: outer (spout < 0), 0: blend
};
struct ROutF {
  double f_rho, f_un, f_ut1, f_ut2, f_eden, f_eint, q_un, q_pres, ustar;
};

CAMR_HD void riemann_fwd(const RIn& in, double gam, const Par& P, RTape& t, ROutF& o) {
  t.wsmall = in.smallc * P.small_dens;
  t.rl = hmax(in.rl, P.small_dens);
  t.pl = hmax(in.pl, P.small_pres);
  t.rr = hmax(in.rr, P.small_dens);
  t.pr = hmax(in.pr, P.small_pres);
  t.wls = std::sqrt(std::fabs(gam * t.pl * t.rl));
  t.wrs = std::sqrt(std::fabs(gam * t.pr * t.rr));
  t.wl = hmax(t.wsmall, t.wls);
  t.wr = hmax(t.wsmall, t.wrs);
  t.den = t.wl + t.wr;
  t.nump = ((t.wr * t.pl + t.wl * t.pr) + t.wl * t.wr * (in.ul - in.ur));
  t.pstar0 = t.nump / t.den;
  t.pstar = hmax(t.pstar0, P.small_pres);
  t.numu = ((t.wl * in.ul + t.wr * in.ur) + (t.pl - t.pr));
  t.ustar0 = t.numu / t.den;
  t.mask0 = std::fabs(t.ustar0) < P.smallu * 0.5 * (std::fabs(in.ul) + std::fabs(in.ur));
  t.ustar = t.mask0 ? 0.0 : t.ustar0;
  double gamco;
  if (t.ustar > 0.) {
    t.sel = 1;
    t.ro_sel = t.rl; t.uo = in.ul; t.po = t.pl; t.reo = in.rel; gamco = gam;
  } else if (t.ustar < 0) {
    t.sel = -1;
    t.ro_sel = t.rr; t.uo = in.ur; t.po = t.pr; t.reo = in.rer; gamco = gam;
  } else {
    t.sel = 0;
    t.ro_sel = 0.5 * (t.rl + t.rr);
    t.uo = 0.5 * (in.ul + in.ur);
    t.po = 0.5 * (t.pl + t.pr);
    t.reo = 0.5 * (in.rel + in.rer);
    gamco = 0.5 * (gam + gam);
  }
  t.ro = hmax(t.ro_sel, P.small_dens);
  t.roinv = 1.0 / t.ro;
  t.co0 = std::sqrt(std::fabs(gamco * t.po * t.roinv));
  t.co = hmax(in.smallc, t.co0);
  t.co2inv = 1.0 / (t.co * t.co);
  t.drho = (t.pstar - t.po) * t.co2inv;
  t.rstar0 = t.ro + t.drho;
  t.rstar = hmax(P.small_dens, t.rstar0);
  t.entho = (t.reo + t.po) * t.roinv * t.co2inv;
  t.estar = t.reo + (t.pstar - t.po) * t.entho;
  t.cstar0 = std::sqrt(std::fabs(gamco * t.pstar / t.rstar));
  t.cstar = hmax(t.cstar0, in.smallc);
  t.sgnm = (t.ustar < 0.) ? -1.0 : 1.0;
  t.spout0 = t.co - t.sgnm * t.uo;
  t.spin0 = t.cstar - t.sgnm * t.ustar;
  const double ushock = 0.5 * (t.spin0 + t.spout0);
  t.shock = (t.pstar - t.po > 0.0);
  t.spin = t.shock ? ushock : t.spin0;
  t.spout = t.shock ? ushock : t.spout0;
  t.scr_zero = (t.spout - t.spin == 0.0);
  t.scr = t.scr_zero ? P.small * in.cav : t.spout - t.spin;
  t.ratio = (t.spout + t.spin) / t.scr;
  t.frac0 = (1.0 + t.ratio) * 0.5;
  t.frac = hmax(0.0, hmin(1.0, t.frac0));
  if (t.ustar > 0.0) {
    t.iv1 = in.vl; t.iv2 = in.v2l;
  } else {
    t.iv1 = in.vr; t.iv2 = in.v2r;
  }
  if (t.ustar == 0.0) {
    t.iv1 = 0.5 * (in.vl + in.vr);
    t.iv2 = 0.5 * (in.v2l + in.v2r);
  }
  if (t.spin >= 0.0) {
    t.wave = 2;
    t.rho_gd = t.rstar; t.iu = t.ustar; t.gdp0 = t.pstar; t.re_gd = t.estar;
  } else if (t.spout < 0.0) {
    t.wave = 1;
    t.rho_gd = t.ro; t.iu = t.uo; t.gdp0 = t.po; t.re_gd = t.reo;
  } else {
    t.wave = 0;
    t.rho_gd = t.frac * t.rstar + (1.0 - t.frac) * t.ro;
    t.iu = t.frac * t.ustar + (1.0 - t.frac) * t.uo;
    t.gdp0 = t.frac * t.pstar + (1.0 - t.frac) * t.po;
    t.re_gd = t.frac * t.estar + (1.0 - t.frac) * t.reo;
  }
  t.gdp = hmax(t.gdp0, P.small_pres);
  t.frho = t.rho_gd * t.iu;
  t.rhoetot = t.re_gd + 0.5 * t.rho_gd * (t.iu * t.iu + t.iv1 * t.iv1 + t.iv2 * t.iv2);
  o.f_rho = t.frho;
  o.f_un = t.frho * t.iu + t.gdp;
  o.f_ut1 = t.frho * t.iv1;
  o.f_ut2 = t.frho * t.iv2;
  o.f_eden = t.iu * (t.rhoetot + t.gdp);
  o.f_eint = t.iu * t.re_gd;
  o.q_un = t.iu;
  o.q_pres = t.gdp;
  o.ustar = t.ustar;
}

// VJP of riemann_fwd: adjoints of the outputs in `bo`, of its inputs out.
CAMR_HD void riemann_vjp(const RIn& in, double gam, const Par& P, const RTape& t,
                         const ROutF& bo, RIn& bi) {
  bi = RIn{0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  double b_iu = bo.q_un, b_gdp = bo.q_pres;
  double b_regd = 0, b_rhogd = 0, b_iv1 = 0, b_iv2 = 0;
  // f_eint = iu*re_gd
  b_iu += bo.f_eint * t.re_gd;
  b_regd += bo.f_eint * t.iu;
  // f_eden = iu*(rhoetot + gdp)
  b_iu += bo.f_eden * (t.rhoetot + t.gdp);
  const double b_rhoetot = bo.f_eden * t.iu;
  b_gdp += bo.f_eden * t.iu;
  // rhoetot = re_gd + 0.5*rho_gd*(iu^2 + iv1^2 + iv2^2)
  b_regd += b_rhoetot;
  const double ss = t.iu * t.iu + t.iv1 * t.iv1 + t.iv2 * t.iv2;
  b_rhogd += b_rhoetot * 0.5 * ss;
  const double hr = 0.5 * t.rho_gd;
  b_iu += b_rhoetot * hr * 2.0 * t.iu;
  b_iv1 += b_rhoetot * hr * 2.0 * t.iv1;
  b_iv2 += b_rhoetot * hr * 2.0 * t.iv2;
  // fluxes through frho
  double b_frho = bo.f_rho;
  b_frho += bo.f_ut2 * t.iv2;
  b_iv2 += bo.f_ut2 * t.frho;
  b_frho += bo.f_ut1 * t.iv1;
  b_iv1 += bo.f_ut1 * t.frho;
  b_frho += bo.f_un * t.iu;
  b_iu += bo.f_un * t.frho;
  b_gdp += bo.f_un;
  b_rhogd += b_frho * t.iu;
  b_iu += b_frho * t.rho_gd;
  // gdp = max(gdp0, small_pres)
  const double b_gdp0 = (t.gdp0 < P.small_pres) ? 0.0 : b_gdp;
  double b_rstar = 0, b_ustar = 0, b_pstar = 0, b_estar = 0;
  double b_ro = 0, b_uo = 0, b_po = 0, b_reo = 0, b_frac = 0;
  if (t.wave == 2) {
    b_rstar += b_rhogd; b_ustar += b_iu; b_pstar += b_gdp0; b_estar += b_regd;
  } else if (t.wave == 1) {
    b_ro += b_rhogd; b_uo += b_iu; b_po += b_gdp0; b_reo += b_regd;
  } else {
    b_frac += b_rhogd * (t.rstar - t.ro) + b_iu * (t.ustar - t.uo) +
              b_gdp0 * (t.pstar - t.po) + b_regd * (t.estar - t.reo);
    b_rstar += b_rhogd * t.frac; b_ro += b_rhogd * (1.0 - t.frac);
    b_ustar += b_iu * t.frac; b_uo += b_iu * (1.0 - t.frac);
    b_pstar += b_gdp0 * t.frac; b_po += b_gdp0 * (1.0 - t.frac);
    b_estar += b_regd * t.frac; b_reo += b_regd * (1.0 - t.frac);
  }
  // transverse velocities
  if (t.ustar == 0.0) {
    bi.vl += 0.5 * b_iv1; bi.vr += 0.5 * b_iv1;
    bi.v2l += 0.5 * b_iv2; bi.v2r += 0.5 * b_iv2;
  } else if (t.ustar > 0.0) {
    bi.vl += b_iv1; bi.v2l += b_iv2;
  } else {
    bi.vr += b_iv1; bi.v2r += b_iv2;
  }
  // frac = max(0, min(1, frac0))
  const double b_frac0 = (t.frac0 < 1.0 && 0.0 < t.frac0) ? b_frac : 0.0;
  const double b_ratio = 0.5 * b_frac0;
  const double iscr = 1.0 / t.scr;
  double b_spout = b_ratio * iscr, b_spin = b_ratio * iscr;
  const double b_scr = -b_ratio * t.ratio * iscr;
  if (t.scr_zero) {
    bi.cav += b_scr * P.small;
  } else {
    b_spout += b_scr;
    b_spin -= b_scr;
  }
  double b_spin0, b_spout0;
  if (t.shock) {
    const double b_ushock = b_spin + b_spout;
    b_spin0 = 0.5 * b_ushock;
    b_spout0 = 0.5 * b_ushock;
  } else {
    b_spin0 = b_spin;
    b_spout0 = b_spout;
  }
  double b_cstar = b_spin0;
  b_ustar += -t.sgnm * b_spin0;
  double b_co = b_spout0;
  b_uo += -t.sgnm * b_spout0;
  // cstar = max(cstar0, smallc)
  double b_cstar0 = 0.0;
  if (t.cstar0 < in.smallc) bi.smallc += b_cstar;
  else b_cstar0 = b_cstar;
  const double gamco = gam;
  if (t.cstar0 > 0.0) {
    const double irs = 1.0 / t.rstar;
    const double B = gamco * t.pstar * irs;
    const double b_B = b_cstar0 * 0.5 / t.cstar0 * sgn(B);
    b_pstar += b_B * gamco * irs;
    b_rstar += -b_B * B * irs;
  }
  // estar = reo + (pstar - po)*entho
  b_reo += b_estar;
  b_pstar += b_estar * t.entho;
  b_po -= b_estar * t.entho;
  const double b_entho = b_estar * (t.pstar - t.po);
  // entho = (reo + po)*roinv*co2inv
  b_reo += b_entho * t.roinv * t.co2inv;
  b_po += b_entho * t.roinv * t.co2inv;
  double b_roinv = b_entho * (t.reo + t.po) * t.co2inv;
  double b_co2inv = b_entho * (t.reo + t.po) * t.roinv;
  // rstar = max(small_dens, rstar0)
  const double b_rstar0 = (P.small_dens < t.rstar0) ? b_rstar : 0.0;
  b_ro += b_rstar0;
  const double b_drho = b_rstar0;
  b_pstar += b_drho * t.co2inv;
  b_po -= b_drho * t.co2inv;
  b_co2inv += b_drho * (t.pstar - t.po);
  // co2inv = 1/(co*co)
  b_co += -2.0 * t.co2inv / t.co * b_co2inv;
  // co = max(smallc, co0)
  double b_co0 = 0.0;
  if (in.smallc < t.co0) b_co0 = b_co;
  else bi.smallc += b_co;
  if (t.co0 > 0.0) {
    const double Cb = gamco * t.po * t.roinv;
    const double b_Cb = b_co0 * 0.5 / t.co0 * sgn(Cb);
    b_po += b_Cb * gamco * t.roinv;
    b_roinv += b_Cb * gamco * t.po;
  }
  b_ro += -b_roinv * t.roinv * t.roinv;
  // ro = max(ro_sel, small_dens)
  const double b_rosel = (t.ro_sel < P.small_dens) ? 0.0 : b_ro;
  double b_rl = 0, b_pl = 0, b_rr = 0, b_pr = 0;
  if (t.sel == 1) {
    b_rl += b_rosel; bi.ul += b_uo; b_pl += b_po; bi.rel += b_reo;
  } else if (t.sel == -1) {
    b_rr += b_rosel; bi.ur += b_uo; b_pr += b_po; bi.rer += b_reo;
  } else {
    b_rl += 0.5 * b_rosel; b_rr += 0.5 * b_rosel;
    bi.ul += 0.5 * b_uo; bi.ur += 0.5 * b_uo;
    b_pl += 0.5 * b_po; b_pr += 0.5 * b_po;
    bi.rel += 0.5 * b_reo; bi.rer += 0.5 * b_reo;
  }
  // ustar = mask0 ? 0 : ustar0
  const double b_ustar0 = t.mask0 ? 0.0 : b_ustar;
  const double iden = 1.0 / t.den;
  const double b_numu = b_ustar0 * iden;
  double b_den = -b_ustar0 * t.ustar0 * iden;
  double b_wl = b_numu * in.ul, b_wr = b_numu * in.ur;
  bi.ul += b_numu * t.wl;
  bi.ur += b_numu * t.wr;
  b_pl += b_numu;
  b_pr -= b_numu;
  // pstar = max(pstar0, small_pres)
  const double b_pstar0 = (t.pstar0 < P.small_pres) ? 0.0 : b_pstar;
  const double b_nump = b_pstar0 * iden;
  b_den += -b_pstar0 * t.pstar0 * iden;
  b_wr += b_nump * t.pl;
  b_pl += b_nump * t.wr;
  b_wl += b_nump * t.pr;
  b_pr += b_nump * t.wl;
  const double du = in.ul - in.ur;
  b_wl += b_nump * t.wr * du;
  b_wr += b_nump * t.wl * du;
  bi.ul += b_nump * t.wl * t.wr;
  bi.ur -= b_nump * t.wl * t.wr;
  b_wl += b_den;
  b_wr += b_den;
  // wl = max(wsmall, wls); wls = sqrt(|gam*pl*rl|)
  double b_wsmall = 0.0;
  double b_wls = 0.0, b_wrs = 0.0;
  if (t.wsmall < t.wls) b_wls = b_wl;
  else b_wsmall += b_wl;
  if (t.wsmall < t.wrs) b_wrs = b_wr;
  else b_wsmall += b_wr;
  if (t.wls > 0.0) {
    const double A = gam * t.pl * t.rl;
    const double b_A = b_wls * 0.5 / t.wls * sgn(A);
    b_pl += b_A * gam * t.rl;
    b_rl += b_A * gam * t.pl;
  }
  if (t.wrs > 0.0) {
    const double A = gam * t.pr * t.rr;
    const double b_A = b_wrs * 0.5 / t.wrs * sgn(A);
    b_pr += b_A * gam * t.rr;
    b_rr += b_A * gam * t.pr;
  }
  bi.smallc += b_wsmall * P.small_dens;
  // clamps of the inputs
  bi.rl += (in.rl < P.small_dens) ? 0.0 : b_rl;
  bi.pl += (in.pl < P.small_pres) ? 0.0 : b_pl;
  bi.rr += (in.rr < P.small_dens) ? 0.0 : b_rr;
  bi.pr += (in.pr < P.small_pres) ? 0.0 : b_pr;
}

// ---------------------------------------------------------------------------
// One interior face of direction d between cells L and R.
struct FaceIn {
  double qL[NQ], qR[NQ];  // primitive records of the two cells
  double sL[NS], sR[NS];  // their slope records in direction d
  double dv[4];           // nodal div u at the face's 4 corners
  double uL[NV], uR[NV];  // conserved states (artificial viscosity)
};
struct FaceOut {
  double f[NV];
  double qpres, qun;
};

// Edge state of one side: sign +1 for the left cell's high face, -1 for
// the right cell's low face.  yq: the right cell's species (the left
// state's fallback quirk, MOL_riemann_K.H:82-86).
struct EdgeTape {
  double rden, enth, a, p0, sd[NSP], sum;
  bool fallback;
};
struct Edge {
  double rho, un, t1, t2, p, re, y[NSP];
};

template <int d>
CAMR_HD void edge_fwd(const double* q, const double* s, const double* yq, double sign,
                      const Par& P, EdgeTape& t, Edge& e) {
  constexpr int un = QU + d;
  constexpr int t1 = (d == 0) ? QV : QU;
  constexpr int t2 = (d == 2) ? QV : QW;
  const double c = q[QC];
  t.rden = hmax(q[QR], P.small_dens);
  t.enth = (q[QRE] + q[QP]) / t.rden;
  t.a = s[S0] + s[S2];
  if (sign > 0) t.p0 = q[QP] + 0.5 * t.a * c;
  else t.p0 = q[QP] - 0.5 * t.a * c;
  e.p = hmax(t.p0, P.small_pres);
  if (sign > 0) {
    e.un = q[un] + 0.5 * ((s[S2] - s[S0]) / q[QR]);
    e.t1 = q[t1] + 0.5 * s[S3];
    e.t2 = q[t2] + 0.5 * s[S4];
  } else {
    e.un = q[un] - 0.5 * ((s[S2] - s[S0]) / q[QR]);
    e.t1 = q[t1] - 0.5 * s[S3];
    e.t2 = q[t2] - 0.5 * s[S4];
  }
  // the quotients by c (NSP + 1) and by the sum (NSP), each group from
  // one reciprocal (rn_div_group: the same bits as the divisions)
  double nq[NSP + 1], qq[NSP + 1];
  for (int sp = 0; sp < NSP; ++sp) nq[sp] = q[QY + sp] * t.a;
  nq[NSP] = t.enth * t.a;
  rn_div_group<NSP + 1>(nq, c, qq);
  double sum = 0.;
  for (int sp = 0; sp < NSP; ++sp) {
    if (sign > 0)
      t.sd[sp] = q[QR] * q[QY + sp] + 0.5 * (s[SY + sp] + qq[sp]);
    else
      t.sd[sp] = q[QR] * q[QY + sp] - 0.5 * (s[SY + sp] + qq[sp]);
    sum += t.sd[sp];
  }
  t.sum = sum;
  t.fallback = sum < P.small_dens;
  double ys[NSP];
  rn_div_group<NSP>(t.sd, sum, ys);
  for (int sp = 0; sp < NSP; ++sp) e.y[sp] = t.fallback ? yq[sp] : ys[sp];
  e.rho = hmax(sum, P.small_dens);
  if (sign > 0) e.re = q[QRE] + 0.5 * (s[SRE] + qq[NSP]);
  else e.re = q[QRE] - 0.5 * (s[SRE] + qq[NSP]);
}

// VJP of edge_fwd: accumulates into bq, bs (this cell) and byq (the cell
// whose species the fallback copies).
template <int d>
CAMR_HD void edge_vjp(const double* q, const double* s, double sign, const Par& P,
                      const EdgeTape& t, const Edge& e, const Edge& be, double* bq, double* bs,
                      double* byq) {
  constexpr int un = QU + d;
  constexpr int t1 = (d == 0) ? QV : QU;
  constexpr int t2 = (d == 2) ? QV : QW;
  const double ic = 1.0 / q[QC];
  const double ic2 = ic * ic;
  const double ir = 1.0 / q[QR];
  const double irden = 1.0 / t.rden;
  double b_a = 0.0, b_c = 0.0, b_enth = 0.0, b_sum = 0.0;
  // re
  bq[QRE] += be.re;
  {
    const double tt = sign * 0.5 * be.re;
    bs[SRE] += tt;
    b_enth += tt * t.a * ic;
    b_a += tt * t.enth * ic;
    b_c += -tt * (t.enth * t.a) * ic2;
  }
  // rho = max(sum, small_dens)
  if (!(t.sum < P.small_dens)) b_sum += be.rho;
  // species
  double b_sd[NSP] = {0.0, 0.0, 0.0};
  if (t.fallback) {
    for (int sp = 0; sp < NSP; ++sp) byq[sp] += be.y[sp];
  } else {
    const double isum = 1.0 / t.sum;
    for (int sp = 0; sp < NSP; ++sp) {
      b_sd[sp] += be.y[sp] * isum;
      b_sum += -be.y[sp] * e.y[sp] * isum;
    }
  }
  for (int sp = 0; sp < NSP; ++sp) {
    const double b = b_sd[sp] + b_sum;
    bq[QR] += b * q[QY + sp];
    bq[QY + sp] += b * q[QR];
    const double tt = sign * 0.5 * b;
    bs[SY + sp] += tt;
    bq[QY + sp] += tt * t.a * ic;
    b_a += tt * q[QY + sp] * ic;
    b_c += -tt * (q[QY + sp] * t.a) * ic2;
  }
  // transverse velocities
  bq[t1] += be.t1;
  bs[S3] += sign * 0.5 * be.t1;
  bq[t2] += be.t2;
  bs[S4] += sign * 0.5 * be.t2;
  // normal velocity
  bq[un] += be.un;
  {
    const double tt = sign * 0.5 * be.un;
    bs[S2] += tt * ir;
    bs[S0] -= tt * ir;
    bq[QR] += -tt * (s[S2] - s[S0]) * ir * ir;
  }
  // p = max(p0, small_pres)
  if (!(t.p0 < P.small_pres)) {
    const double b = be.p;
    bq[QP] += b;
    b_a += sign * 0.5 * b * q[QC];
    b_c += sign * 0.5 * b * t.a;
  }
  // enth = (re + p)/max(rho, small_dens)
  bq[QRE] += b_enth * irden;
  bq[QP] += b_enth * irden;
  if (!(q[QR] < P.small_dens)) bq[QR] += -b_enth * t.enth * irden;
  bs[S0] += b_a;
  bs[S2] += b_a;
  bq[QC] += b_c;
}

struct FaceTape {
  EdgeTape tl, tr;
  Edge el, er;
  RIn rin;
  RTape rt;
  ROutF ro;
  double f0[NV];  // fluxes before adjust_fluxes
  double f1[NV];  // after artificial viscosity
  double div, dsum, summ, fac;
};

template <int d>
CAMR_HD void face_forward(const FaceIn& in, double dx, double area, const Par& P,
                          FaceTape& t, FaceOut& out) {
  edge_fwd<d>(in.qL, in.sL, in.qR + QY, 1.0, P, t.tl, t.el);
  edge_fwd<d>(in.qR, in.sR, in.qR + QY, -1.0, P, t.tr, t.er);
  t.rin.rl = t.el.rho; t.rin.ul = t.el.un; t.rin.vl = t.el.t1; t.rin.v2l = t.el.t2;
  t.rin.pl = t.el.p; t.rin.rel = t.el.re;
  t.rin.rr = t.er.rho; t.rin.ur = t.er.un; t.rin.vr = t.er.t1; t.rin.v2r = t.er.t2;
  t.rin.pr = t.er.p; t.rin.rer = t.er.re;
  t.rin.cav = 0.5 * (in.qR[QC] + in.qL[QC]);
  t.rin.smallc = hmax(in.qR[QCS], in.qL[QCS]);
  riemann_fwd(t.rin, P.gamma, P, t.rt, t.ro);
  constexpr int fu = MX + d;
  constexpr int fv = (d == 0) ? MY : MX;
  constexpr int fv2 = (d == 2) ? MY : MZ;
  double* f = t.f0;
  f[RHO] = t.ro.f_rho;
  f[fu] = t.ro.f_un;
  f[fv] = t.ro.f_ut1;
  f[fv2] = t.ro.f_ut2;
  f[EDEN] = t.ro.f_eden;
  f[EINT] = t.ro.f_eint;
  f[TEMP] = 0.0;
  for (int sp = 0; sp < NSP; ++sp) {
    if (t.ro.ustar > 0.0) f[FS + sp] = t.ro.f_rho * t.el.y[sp];
    else if (t.ro.ustar < 0.0) f[FS + sp] = t.ro.f_rho * t.er.y[sp];
    else f[FS + sp] = t.ro.f_rho * 0.50 * (t.el.y[sp] + t.er.y[sp]);
  }
  // adjust_fluxes (interior face)
  t.dsum = 0.25 * (in.dv[0] + in.dv[1] + in.dv[2] + in.dv[3]);
  t.div = P.difmag * hmin(0.0, t.dsum);
  for (int n = 0; n < NV; ++n) {
    t.f1[n] = f[n];
    if (n != TEMP) t.f1[n] += dx * t.div * (in.uR[n] - in.uL[n]);
  }
  t.f1[TEMP] = 0.0;
  double summ = 0.0;
  for (int n = FS; n < FS + NSP; ++n) summ += t.f1[n];
  t.summ = summ;
  t.fac = (summ != 0.0) ? t.f1[RHO] / summ : 1.0;
  for (int n = 0; n < NV; ++n) {
    double v = t.f1[n];
    if (n >= FS) v *= t.fac;
    out.f[n] = v * area;
  }
  out.qpres = t.ro.q_pres;
  out.qun = t.ro.q_un;
}

// VJP of face_forward: bout -> bin (accumulated).
template <int d>
CAMR_HD void face_vjp(const FaceIn& in, double dx, double area, const Par& P,
                      const FaceTape& t, const FaceOut& bout, FaceIn& bin) {
  double b_f1[NV], b_f0[NV];
  double b_fac = 0.0;
  for (int n = 0; n < NV; ++n) {
    const double b2 = bout.f[n] * area;
    if (n >= FS) {
      b_f1[n] = b2 * t.fac;
      b_fac += b2 * t.f1[n];
    } else {
      b_f1[n] = b2;
    }
  }
  if (t.summ != 0.0) {
    const double isumm = 1.0 / t.summ;
    b_f1[RHO] += b_fac * isumm;
    const double b_summ = -b_fac * t.fac * isumm;
    for (int n = FS; n < FS + NSP; ++n) b_f1[n] += b_summ;
  }
  b_f1[TEMP] = 0.0;
  double b_div = 0.0;
  for (int n = 0; n < NV; ++n) {
    b_f0[n] = b_f1[n];
    if (n == TEMP) continue;
    b_div += b_f1[n] * dx * (in.uR[n] - in.uL[n]);
    bin.uR[n] += b_f1[n] * dx * t.div;
    bin.uL[n] -= b_f1[n] * dx * t.div;
  }
  if (t.dsum < 0.0) {
    const double b = b_div * P.difmag * 0.25;
    for (int c = 0; c < 4; ++c) bin.dv[c] += b;
  }
  // species fluxes
  constexpr int fu = MX + d;
  constexpr int fv = (d == 0) ? MY : MX;
  constexpr int fv2 = (d == 2) ? MY : MZ;
  ROutF bro{0, 0, 0, 0, 0, 0, 0, 0, 0};
  Edge bel{0, 0, 0, 0, 0, 0, {0, 0, 0}}, ber{0, 0, 0, 0, 0, 0, {0, 0, 0}};
  for (int sp = 0; sp < NSP; ++sp) {
    const double b = b_f0[FS + sp];
    if (t.ro.ustar > 0.0) {
      bro.f_rho += b * t.el.y[sp];
      bel.y[sp] += b * t.ro.f_rho;
    } else if (t.ro.ustar < 0.0) {
      bro.f_rho += b * t.er.y[sp];
      ber.y[sp] += b * t.ro.f_rho;
    } else {
      bro.f_rho += b * 0.5 * (t.el.y[sp] + t.er.y[sp]);
      bel.y[sp] += b * t.ro.f_rho * 0.5;
      ber.y[sp] += b * t.ro.f_rho * 0.5;
    }
  }
  bro.f_rho += b_f0[RHO];
  bro.f_un = b_f0[fu];
  bro.f_ut1 = b_f0[fv];
  bro.f_ut2 = b_f0[fv2];
  bro.f_eden = b_f0[EDEN];
  bro.f_eint = b_f0[EINT];
  bro.q_pres = bout.qpres;
  bro.q_un = bout.qun;
  RIn bri;
  riemann_vjp(t.rin, P.gamma, P, t.rt, bro, bri);
  bel.rho += bri.rl; bel.un += bri.ul; bel.t1 += bri.vl; bel.t2 += bri.v2l;
  bel.p += bri.pl; bel.re += bri.rel;
  ber.rho += bri.rr; ber.un += bri.ur; ber.t1 += bri.vr; ber.t2 += bri.v2r;
  ber.p += bri.pr; ber.re += bri.rer;
  bin.qR[QC] += 0.5 * bri.cav;
  bin.qL[QC] += 0.5 * bri.cav;
  if (in.qR[QCS] < in.qL[QCS]) bin.qL[QCS] += bri.smallc;
  else bin.qR[QCS] += bri.smallc;
  edge_vjp<d>(in.qR, in.sR, -1.0, P, t.tr, t.er, ber, bin.qR, bin.sR, bin.qR + QY);
  edge_vjp<d>(in.qL, in.sL, 1.0, P, t.tl, t.el, bel, bin.qL, bin.sL, bin.qR + QY);
}

// ---------------------------------------------------------------------------
// MC limiter and the slopes of one cell in direction d from the primitive
// records of cells c-1, c, c+1.
struct LimTape {
  double dl, dr, dcen, slop;
  int which;  // 0: |dcen|; 1: theta*|dl|; 2: theta*|dr|; 3: zero (dl*dr < 0)
};

CAMR_HD double limiter_fwd(double dl, double dr, LimTape& t) {
  const double theta = 2.0;
  t.dl = dl;
  t.dr = dr;
  t.dcen = 0.5 * (dl + dr);
  const double dsgn = std::copysign(1.0, t.dcen);
  const double mn = hmin(std::fabs(dl), std::fabs(dr));
  t.slop = theta * mn;
  const double dlim = (dl * dr >= 0.0) ? t.slop : 0.0;
  const double fc = std::fabs(t.dcen);
  const double r = dsgn * hmin(dlim, fc);
  if (fc < dlim) t.which = 0;
  else if (!(dl * dr >= 0.0)) t.which = 3;
  else t.which = (std::fabs(dr) < std::fabs(dl)) ? 2 : 1;
  return r;
}

CAMR_HD void limiter_vjp(const LimTape& t, double b, double& bdl, double& bdr) {
  const double dsgn = std::copysign(1.0, t.dcen);
  const double theta = 2.0;
  if (t.which == 0) {
    // dsgn * |dcen| = dcen
    bdl += 0.5 * b;
    bdr += 0.5 * b;
  } else if (t.which == 1) {
    bdl += b * dsgn * theta * dabs(t.dl);
  } else if (t.which == 2) {
    bdr += b * dsgn * theta * dabs(t.dr);
  }
}

struct SlopeTape {
  LimTape lt[NS];
  double rden, enth, cs2;
};

template <int d>
CAMR_HD void slope_fwd(const double* qm, const double* q0, const double* qp, const Par& P,
                       SlopeTape& t, double* o) {
  constexpr int un = QU + d;
  constexpr int t1 = (d == 0) ? QV : QU;
  constexpr int t2 = (d == 2) ? QV : QW;
  const double c = q0[QC];
  t.cs2 = c * c;
  t.rden = hmax(q0[QR], P.small_dens);
  t.enth = (q0[QRE] + q0[QP]) / t.rden;
  const double dpl = q0[QP] - qm[QP], dpr = qp[QP] - q0[QP];
  // the quotients by c (2) and by c^2 (2 + 2 NSP), each group from one
  // reciprocal (rn_div_group: the same bits as the divisions)
  const double nc[2] = {0.5 * dpl, 0.5 * dpr};
  double qc[2];
  rn_div_group<2>(nc, c, qc);
  double ns[2 + 2 * NSP], qs[2 + 2 * NSP];
  ns[0] = t.enth * dpl;
  ns[1] = t.enth * dpr;
  for (int sp = 0; sp < NSP; ++sp) {
    ns[2 + 2 * sp] = q0[QY + sp] * dpl;
    ns[3 + 2 * sp] = q0[QY + sp] * dpr;
  }
  rn_div_group<2 + 2 * NSP>(ns, t.cs2, qs);
  double dl = qc[0] - 0.5 * q0[QR] * (q0[un] - qm[un]);
  double dr = qc[1] - 0.5 * q0[QR] * (qp[un] - q0[un]);
  o[S0] = limiter_fwd(dl, dr, t.lt[S0]);
  dl = qc[0] + 0.5 * q0[QR] * (q0[un] - qm[un]);
  dr = qc[1] + 0.5 * q0[QR] * (qp[un] - q0[un]);
  o[S2] = limiter_fwd(dl, dr, t.lt[S2]);
  o[S3] = limiter_fwd(q0[t1] - qm[t1], qp[t1] - q0[t1], t.lt[S3]);
  o[S4] = limiter_fwd(q0[t2] - qm[t2], qp[t2] - q0[t2], t.lt[S4]);
  dl = (q0[QRE] - qm[QRE]) - qs[0];
  dr = (qp[QRE] - q0[QRE]) - qs[1];
  o[SRE] = limiter_fwd(dl, dr, t.lt[SRE]);
  for (int sp = 0; sp < NSP; ++sp) {
    const int n = QY + sp;
    dl = q0[QR] * q0[n] - qm[QR] * qm[n] - qs[2 + 2 * sp];
    dr = qp[QR] * qp[n] - q0[QR] * q0[n] - qs[3 + 2 * sp];
    o[SY + sp] = limiter_fwd(dl, dr, t.lt[SY + sp]);
  }
}

template <int d>
CAMR_HD void slope_vjp(const double* qm, const double* q0, const double* qp, const Par& P,
                       const SlopeTape& t, const double* bo, double* bqm, double* bq0,
                       double* bqp) {
  constexpr int un = QU + d;
  constexpr int t1 = (d == 0) ? QV : QU;
  constexpr int t2 = (d == 2) ? QV : QW;
  const double c = q0[QC];
  const double ic = 1.0 / c;
  const double ics2 = 1.0 / t.cs2;
  const double ics4 = ics2 * ics2;
  const double irden = 1.0 / t.rden;
  double b_c = 0.0, b_cs2 = 0.0, b_enth = 0.0;
  // species
  for (int sp = 0; sp < NSP; ++sp) {
    const int n = QY + sp;
    double bdl = 0.0, bdr = 0.0;
    limiter_vjp(t.lt[SY + sp], bo[SY + sp], bdl, bdr);
    // dl = r0*y0 - rm*ym - y0*(p0-pm)/cs2
    bq0[QR] += bdl * q0[n];
    bq0[n] += bdl * q0[QR];
    bqm[QR] -= bdl * qm[n];
    bqm[n] -= bdl * qm[QR];
    bq0[n] -= bdl * (q0[QP] - qm[QP]) * ics2;
    bq0[QP] -= bdl * q0[n] * ics2;
    bqm[QP] += bdl * q0[n] * ics2;
    b_cs2 += bdl * q0[n] * (q0[QP] - qm[QP]) * ics4;
    // dr = rp*yp - r0*y0 - y0*(pp-p0)/cs2
    bqp[QR] += bdr * qp[n];
    bqp[n] += bdr * qp[QR];
    bq0[QR] -= bdr * q0[n];
    bq0[n] -= bdr * q0[QR];
    bq0[n] -= bdr * (qp[QP] - q0[QP]) * ics2;
    bqp[QP] -= bdr * q0[n] * ics2;
    bq0[QP] += bdr * q0[n] * ics2;
    b_cs2 += bdr * q0[n] * (qp[QP] - q0[QP]) * ics4;
  }
  {
    double bdl = 0.0, bdr = 0.0;
    limiter_vjp(t.lt[SRE], bo[SRE], bdl, bdr);
    bq0[QRE] += bdl;
    bqm[QRE] -= bdl;
    b_enth -= bdl * (q0[QP] - qm[QP]) * ics2;
    bq0[QP] -= bdl * t.enth * ics2;
    bqm[QP] += bdl * t.enth * ics2;
    b_cs2 += bdl * t.enth * (q0[QP] - qm[QP]) * ics4;
    bqp[QRE] += bdr;
    bq0[QRE] -= bdr;
    b_enth -= bdr * (qp[QP] - q0[QP]) * ics2;
    bqp[QP] -= bdr * t.enth * ics2;
    bq0[QP] += bdr * t.enth * ics2;
    b_cs2 += bdr * t.enth * (qp[QP] - q0[QP]) * ics4;
    bq0[QRE] += b_enth * irden;
    bq0[QP] += b_enth * irden;
    if (!(q0[QR] < P.small_dens)) bq0[QR] += -b_enth * t.enth * irden;
  }
  {
    double bdl = 0.0, bdr = 0.0;
    limiter_vjp(t.lt[S4], bo[S4], bdl, bdr);
    bq0[t2] += bdl - bdr;
    bqm[t2] -= bdl;
    bqp[t2] += bdr;
  }
  {
    double bdl = 0.0, bdr = 0.0;
    limiter_vjp(t.lt[S3], bo[S3], bdl, bdr);
    bq0[t1] += bdl - bdr;
    bqm[t1] -= bdl;
    bqp[t1] += bdr;
  }
  for (int w = 0; w < 2; ++w) {
    const double sg = (w == 0) ? -1.0 : 1.0;  // S0: minus, S2: plus
    double bdl = 0.0, bdr = 0.0;
    limiter_vjp(t.lt[w == 0 ? S0 : S2], bo[w == 0 ? S0 : S2], bdl, bdr);
    // dl = 0.5*(p0-pm)/c + sg*0.5*r0*(u0-um)
    bq0[QP] += bdl * 0.5 * ic;
    bqm[QP] -= bdl * 0.5 * ic;
    b_c += -bdl * 0.5 * (q0[QP] - qm[QP]) * ic * ic;
    bq0[QR] += bdl * sg * 0.5 * (q0[un] - qm[un]);
    bq0[un] += bdl * sg * 0.5 * q0[QR];
    bqm[un] -= bdl * sg * 0.5 * q0[QR];
    bqp[QP] += bdr * 0.5 * ic;
    bq0[QP] -= bdr * 0.5 * ic;
    b_c += -bdr * 0.5 * (qp[QP] - q0[QP]) * ic * ic;
    bq0[QR] += bdr * sg * 0.5 * (qp[un] - q0[un]);
    bqp[un] += bdr * sg * 0.5 * q0[QR];
    bq0[un] -= bdr * sg * 0.5 * q0[QR];
  }
  b_c += b_cs2 * 2.0 * c;
  bq0[QC] += b_c;
}

// ---------------------------------------------------------------------------
// hydro_ctoprim of one cell (U -> q) and its VJP.
CAMR_HD void ctoprim_fwd(const double* u, const Par& P, double* q, bool& eint_branch) {
  const double rho = u[RHO];
  const double rhoinv = 1.0 / rho;
  const double vx = u[MX] * rhoinv, vy = u[MY] * rhoinv, vz = u[MZ] * rhoinv;
  const double kineng = 0.5 * rho * (vx * vx + vy * vy + vz * vz);
  double e;
  eint_branch = !((u[EDEN] - kineng) / u[EDEN] > P.eta1);
  if (!eint_branch) e = (u[EDEN] - kineng) * rhoinv;
  else e = u[EINT] * rhoinv;
  q[QR] = rho;
  q[QU] = vx;
  q[QV] = vy;
  q[QW] = vz;
  q[QP] = (P.gamma - 1.0) * rho * e;
  q[QRE] = e * rho;
  for (int sp = 0; sp < NSP; ++sp) q[QY + sp] = u[FS + sp] * rhoinv;
  q[QC] = std::sqrt(P.gamma * q[QP] / rho);
  q[QCS] = hmax(P.small_num, P.small_num * q[QC]);
}

CAMR_HD void ctoprim_vjp(const double* u, const Par& P, const double* bq, double* bu) {
  double q[NQ];
  bool eint_branch;
  ctoprim_fwd(u, P, q, eint_branch);
  const double rho = u[RHO];
  const double rhoinv = 1.0 / rho;
  double b_rho = bq[QR], b_rhoinv = 0.0;
  double b_c = bq[QC];
  if (P.small_num < P.small_num * q[QC]) b_c += bq[QCS] * P.small_num;
  double b_p = bq[QP];
  if (q[QC] > 0.0) {
    const double X = P.gamma * q[QP] / rho;
    const double b_X = b_c * 0.5 / q[QC];
    b_p += b_X * P.gamma / rho;
    b_rho += -b_X * X / rho;
  }
  const double vx0 = u[MX] * rhoinv, vy0 = u[MY] * rhoinv, vz0 = u[MZ] * rhoinv;
  const double kin0 = 0.5 * rho * (vx0 * vx0 + vy0 * vy0 + vz0 * vz0);
  const double e = eint_branch ? u[EINT] * rhoinv : (u[EDEN] - kin0) * rhoinv;
  // rhoe = e*rho ; p = (gamma-1)*rho*e
  double b_e = bq[QRE] * rho + b_p * (P.gamma - 1.0) * rho;
  b_rho += bq[QRE] * e + b_p * (P.gamma - 1.0) * e;
  for (int sp = 0; sp < NSP; ++sp) {
    bu[FS + sp] += bq[QY + sp] * rhoinv;
    b_rhoinv += bq[QY + sp] * u[FS + sp];
  }
  double b_vx = bq[QU], b_vy = bq[QV], b_vz = bq[QW];
  const double vx = u[MX] * rhoinv, vy = u[MY] * rhoinv, vz = u[MZ] * rhoinv;
  if (eint_branch) {
    bu[EINT] += b_e * rhoinv;
    b_rhoinv += b_e * u[EINT];
  } else {
    const double kineng = 0.5 * rho * (vx * vx + vy * vy + vz * vz);
    bu[EDEN] += b_e * rhoinv;
    const double b_kin = -b_e * rhoinv;
    b_rhoinv += b_e * (u[EDEN] - kineng);
    b_rho += b_kin * 0.5 * (vx * vx + vy * vy + vz * vz);
    b_vx += b_kin * rho * vx;
    b_vy += b_kin * rho * vy;
    b_vz += b_kin * rho * vz;
  }
  bu[MX] += b_vx * rhoinv;
  bu[MY] += b_vy * rhoinv;
  bu[MZ] += b_vz * rhoinv;
  b_rhoinv += b_vx * u[MX] + b_vy * u[MY] + b_vz * u[MZ];
  b_rho += -b_rhoinv * rhoinv * rhoinv;
  bu[RHO] += b_rho;
}

// ---------------------------------------------------------------------------
// clean_state of a valid cell without a density reset: normalize_species,
// then computeTemp's reset_internal_energy (allow_small_energy = 1,
// allow_negative_energy = 0 branch) and T.  UTEMP feeds no other state
// variable, so its adjoint is dropped.
struct CleanTape {
  double ain[NSP], m[NSP], y[NSP], sum, sum2;
  bool norm;
  double rho, mx, my, mz, ueden, ueint;  // after normalisation
  int branch;  // 0: E<0 ; 1: eint = E - rho ke ; 2: E = eint + rho ke ; 3: small eint ; 4: none
  bool small_e_reset;  // branch 0: eint reset from small T
};

CAMR_HD double rty2e(double gamma, double T, const double* y) {
  const double RU = 8.31446261815324e7, AIRMW = 26.93;
  const double cv = RU / (AIRMW * (gamma - 1.0));
  double e = 0.0;
  for (int n = 0; n < NSP; ++n) e += y[n] * (cv * T);
  return e;
}

CAMR_HD void clean_fwd(const double* s_in, const Par& P, CleanTape& t, double* s) {
  for (int n = 0; n < NV; ++n) s[n] = s_in[n];
  double sum = 0.;
  for (int sp = 0; sp < NSP; ++sp) {
    t.ain[sp] = s[FS + sp];
    t.m[sp] = hmin(s[RHO], t.ain[sp]);
    t.y[sp] = hmax(t.m[sp], 0.0);
    s[FS + sp] = t.y[sp];
    sum += s[FS + sp];
  }
  t.sum = sum;
  t.norm = s[RHO] > 0.;
  if (t.norm) {
    t.sum2 = sum / s[RHO];
    for (int sp = 0; sp < NSP; ++sp) s[FS + sp] /= t.sum2;
  }
  const double rho = s[RHO];
  const double rhoInv = 1.0 / rho;
  const double Up = s[MX] * rhoInv, Vp = s[MY] * rhoInv, Wp = s[MZ] * rhoInv;
  const double ke = 0.5 * (Up * Up + Vp * Vp + Wp * Wp);
  t.rho = rho; t.mx = s[MX]; t.my = s[MY]; t.mz = s[MZ]; t.ueden = s[EDEN]; t.ueint = s[EINT];
  double mf[NSP];
  for (int sp = 0; sp < NSP; ++sp) mf[sp] = s[FS + sp] * rhoInv;
  t.small_e_reset = false;
  if (s[EDEN] < 0.) {
    t.branch = 0;
    if (s[EINT] < 0.) {
      t.small_e_reset = true;
      s[EINT] = rho * rty2e(P.gamma, P.small_temp, mf);
    }
    s[EDEN] = s[EINT] + rho * ke;
  } else {
    const double rho_eint = s[EDEN] - s[RHO] * ke;
    if (rho_eint > 0. && rho_eint / s[EDEN] > P.eta2) {
      t.branch = 1;
      s[EINT] = rho_eint;
    } else if (s[EINT] > 0 && P.dual_energy_update_E_from_e == 1) {
      t.branch = 2;
      s[EDEN] = s[EINT] + rho * ke;
    } else if (s[EINT] <= 0.) {
      t.branch = 3;
      const double e_out = rty2e(P.gamma, P.small_temp, mf);
      s[EINT] = rho * e_out;
      if (P.dual_energy_update_E_from_e == 1) s[EDEN] += (rho * e_out - s[EINT]);
    } else {
      t.branch = 4;
    }
  }
  const double RU = 8.31446261815324e7, AIRMW = 26.93;
  s[TEMP] = (P.gamma - 1.0) * (s[EINT] * (1.0 / s[RHO])) * AIRMW / RU;
}

CAMR_HD void clean_vjp(const double* s_in, const Par& P, const double* bs_out, double* bs_in) {
  CleanTape t;
  double s[NV];
  clean_fwd(s_in, P, t, s);
  double b[NV];
  for (int n = 0; n < NV; ++n) b[n] = bs_out[n];
  b[TEMP] = 0.0;
  const double rho = t.rho;
  const double rhoInv = 1.0 / rho;
  const double Up = t.mx * rhoInv, Vp = t.my * rhoInv, Wp = t.mz * rhoInv;
  const double ke = 0.5 * (Up * Up + Vp * Vp + Wp * Wp);
  double b_rho = 0.0, b_ke = 0.0;
  double b_fs[NSP] = {0.0, 0.0, 0.0};
  for (int sp = 0; sp < NSP; ++sp) b_fs[sp] = b[FS + sp];
  double b_eden = b[EDEN], b_eint = b[EINT];
  auto small_e_vjp = [&](double b_out_eint) {
    // EINT = rho * rty2e(small_T, FS/rho): linear in the species, rho cancels
    const double RU = 8.31446261815324e7, AIRMW = 26.93;
    const double cvT = RU / (AIRMW * (P.gamma - 1.0)) * P.small_temp;
    for (int sp = 0; sp < NSP; ++sp) b_fs[sp] += b_out_eint * cvT;
  };
  if (t.branch == 0) {
    // EDEN = EINT + rho*ke
    b_eint += b_eden;
    b_rho += b_eden * ke;
    b_ke += b_eden * rho;
    b_eden = 0.0;
    if (t.small_e_reset) {
      small_e_vjp(b_eint);
      b_eint = 0.0;
    }
  } else if (t.branch == 1) {
    // EINT = EDEN - rho*ke
    b_eden += b_eint;
    b_rho += -b_eint * ke;
    b_ke += -b_eint * rho;
    b_eint = 0.0;
  } else if (t.branch == 2) {
    b_eint += b_eden;
    b_rho += b_eden * ke;
    b_ke += b_eden * rho;
    b_eden = 0.0;
  } else if (t.branch == 3) {
    // EDEN += rho*e_out - EINT_new with EINT_new = rho*e_out: EDEN unchanged
    small_e_vjp(b_eint);
    b_eint = 0.0;
  }
  // ke = 0.5*(U^2+V^2+W^2), U = mx/rho
  double b_mx = b[MX] + b_ke * Up * rhoInv, b_my = b[MY] + b_ke * Vp * rhoInv,
         b_mz = b[MZ] + b_ke * Wp * rhoInv;
  b_rho += -b_ke * (Up * Up + Vp * Vp + Wp * Wp) * rhoInv;
  b_rho += b[RHO];
  // normalize_species
  if (t.norm) {
    double b_sum2 = 0.0;
    for (int sp = 0; sp < NSP; ++sp) {
      const double outv = t.y[sp] / t.sum2;
      b_sum2 += -b_fs[sp] * outv / t.sum2;
      b_fs[sp] = b_fs[sp] / t.sum2;
    }
    const double b_sum = b_sum2 / rho;
    b_rho += -b_sum2 * t.sum2 / rho;
    for (int sp = 0; sp < NSP; ++sp) b_fs[sp] += b_sum;
  }
  for (int sp = 0; sp < NSP; ++sp) {
    const double b_m = (t.m[sp] < 0.0) ? 0.0 : b_fs[sp];
    if (t.ain[sp] < s_in[RHO]) bs_in[FS + sp] += b_m;
    else b_rho += b_m;
  }
  bs_in[RHO] += b_rho;
  bs_in[MX] += b_mx;
  bs_in[MY] += b_my;
  bs_in[MZ] += b_mz;
  bs_in[EDEN] += b_eden;
  bs_in[EINT] += b_eint;
}

}  // namespace adj
}  // namespace camr
