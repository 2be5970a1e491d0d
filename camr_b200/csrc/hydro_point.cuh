// Pointwise FP64 device functions of the hydro advance.  Each one reproduces
// the reference's arithmetic operation by operation (same operands, same
// order; the library is compiled with -fmad=false), so results match the
// reference CPU build bit for bit.  States live in registers as ES_* records
// (rho, u, v, w, p, rho*e, 3 species), velocities in absolute (x, y, z)
// order as in the reference's QVAR arrays.
#pragma once

#include "camr_common.cuh"

namespace camr {

struct CellAux {
  double c, csml, gamc;  // qaux QC, QCSML, QGAMC
};

// Riemann solver outputs (Source/Hydro/Hydro_riemann.H:8-173).
struct ROut {
  double ustar;
  double f_rho, f_un, f_ut1, f_ut2, f_eden, f_eint;
  double q_un, q_pres;
};

__device__ __forceinline__ ROut riemannus(double rl_in, double ul, double vl, double v2l,
                                          double pl_in, double rel, double rr_in, double ur,
                                          double vr, double v2r, double pr_in, double rer,
                                          double cav, double gamcl, double gamcr,
                                          double small, double smallc, double small_dens,
                                          double small_pres, double smallu) {
  ROut o;
  const double wsmall = smallc * small_dens;
  const double rl = dmax(rl_in, small_dens);
  const double pl = dmax(pl_in, small_pres);
  const double rr = dmax(rr_in, small_dens);
  const double pr = dmax(pr_in, small_pres);
  const double wl = dmax(wsmall, sqrt(fabs(gamcl * pl * rl)));
  const double wr = dmax(wsmall, sqrt(fabs(gamcr * pr * rr)));
  double pstar = ((wr * pl + wl * pr) + wl * wr * (ul - ur)) / (wl + wr);
  pstar = dmax(pstar, small_pres);
  double ustar = ((wl * ul + wr * ur) + (pl - pr)) / (wl + wr);
  bool mask = fabs(ustar) < smallu * 0.5 * (fabs(ul) + fabs(ur));
  ustar = mask ? 0.0 : ustar;
  // upwind state (left, right, or the mean when ustar is exactly 0),
  // picked by selects rather than branches: the same values, fewer
  // divergent branches
  const bool up = ustar > 0., dn = ustar < 0;
  double ro = up ? rl : dn ? rr : 0.5 * (rl + rr);
  const double uo = up ? ul : dn ? ur : 0.5 * (ul + ur);
  const double po = up ? pl : dn ? pr : 0.5 * (pl + pr);
  const double reo = up ? rel : dn ? rer : 0.5 * (rel + rer);
  const double gamco = up ? gamcl : dn ? gamcr : 0.5 * (gamcl + gamcr);
  ro = dmax(ro, small_dens);
  const double roinv = 1.0 / ro;
  double co = sqrt(fabs(gamco * po * roinv));
  co = dmax(smallc, co);
  const double co2inv = 1.0 / (co * co);
  const double drho = (pstar - po) * co2inv;
  double rstar = ro + drho;
  rstar = dmax(small_dens, rstar);
  const double entho = (reo + po) * roinv * co2inv;
  const double estar = reo + (pstar - po) * entho;
  double cstar = sqrt(fabs(gamco * pstar / rstar));
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
  o.q_pres = qint_gdpres;
  return o;
}

// HLLC approximate Riemann solver (riemann_solver = 1; not in the
// reference, which has only riemannus).  Toro, "Riemann Solvers and
// Numerical Methods for Fluid Dynamics", 3rd ed., sec. 10.4-10.6: Davis
// wave-speed estimates S_L = min(u_L - c_L, u_R - c_R), S_R = max(u_L + c_L,
// u_R + c_R); contact speed S* from the two star-momentum balances; the flux
// of the region containing x/t = 0 (F_L, F_L + S_L (U*_L - U_L),
// F_R + S_R (U*_R - U_R), F_R).  rho e travels like a passive density.
// Returned interface values: the normal velocity and pressure of that region
// (S*, p* = p_L + rho_L (S_L - u_L)(S* - u_L) in the star regions).
__device__ __forceinline__ ROut hllc(double rl_in, double ul, double vl, double v2l,
                                     double pl_in, double rel, double rr_in, double ur,
                                     double vr, double v2r, double pr_in, double rer,
                                     double gamcl, double gamcr, double smallc,
                                     double small_dens, double small_pres) {
  ROut o;
  const double rl = dmax(rl_in, small_dens);
  const double pl = dmax(pl_in, small_pres);
  const double rr = dmax(rr_in, small_dens);
  const double pr = dmax(pr_in, small_pres);
  const double cl = dmax(smallc, sqrt(fabs(gamcl * pl / rl)));
  const double cr = dmax(smallc, sqrt(fabs(gamcr * pr / rr)));
  const double sl = dmin(ul - cl, ur - cr);
  const double sr = dmax(ul + cl, ur + cr);
  const double el = rel + 0.5 * rl * (ul * ul + vl * vl + v2l * v2l);
  const double er = rer + 0.5 * rr * (ur * ur + vr * vr + v2r * v2r);
  const double dl = rl * (sl - ul);
  const double dr = rr * (sr - ur);
  const double sstar = ((pr - pl) + (ul * dl - ur * dr)) / (dl - dr);
  const double pstar = pl + dl * (sstar - ul);
  // the side whose states enter the flux
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
  o.q_pres = dmax(q_pres, small_pres);
  return o;
}

// Full conserved flux of one face plus the interface pressure and normal
// velocity.  Source/Hydro/Hydro_cmpflx.H:153-311.  ql/qr are modified in
// place at a physical-boundary face exactly as the reference modifies its
// state arrays (:239-282).  f[UTEMP] is left at 0 (flux arrays start from
// setVal(0), CAMR_construct_hydro_source.cpp:88).
//
// cmpflx_core does all but the species: the boundary edits, the Riemann
// solve and every non-species flux component; species_flux then upwinds the
// species edge states by the sign of ustar.
template <int dir>
__device__ __forceinline__ ROut cmpflx_core(double* ql, double* qr, const CellAux& aL,
                                            const CellAux& aR, int idx, int bclo, int bchi,
                                            int domlo, int domhi, const KParams& P,
                                            double* f) {
  constexpr int iu = ES_U + dir;
  constexpr int iv = (dir == 0) ? ES_V : ES_U;
  constexpr int iv2 = (dir == 2) ? ES_V : ES_W;
  const double cav = 0.5 * (aR.c + aL.c);
  const double smallc = dmax(aR.csml, aL.csml);
  double gamcl = aL.gamc;
  double gamcr = aR.gamc;
  double ul = ql[iu], vl = ql[iv], v2l = ql[iv2];
  double ur = qr[iu], vr = qr[iv], v2r = qr[iv2];
  if (idx == domlo) {
    if (bclo == CAMR_BC_SYMMETRY || bclo == CAMR_BC_SLIPWALL || bclo == CAMR_BC_NOSLIPWALL) {
      ql[ES_RHO] = qr[ES_RHO];
      ql[ES_P] = qr[ES_P];
      ql[ES_REINT] = qr[ES_REINT];
      gamcl = gamcr;
      ul = -ur;
      vl = vr;
      v2l = v2r;
    } else if (bclo == CAMR_BC_OUTFLOW) {
      ul = ur;
      vl = vr;
      v2l = v2r;
      gamcl = gamcr;
      ql[ES_RHO] = qr[ES_RHO];
      ql[ES_P] = qr[ES_P];
      ql[ES_REINT] = qr[ES_REINT];
    }
  }
  if (idx == domhi + 1) {
    if (bchi == CAMR_BC_SYMMETRY || bchi == CAMR_BC_SLIPWALL || bchi == CAMR_BC_NOSLIPWALL) {
      qr[ES_RHO] = ql[ES_RHO];
      qr[ES_P] = ql[ES_P];
      qr[ES_REINT] = ql[ES_REINT];
      gamcr = gamcl;
      ur = -ul;
      vr = vl;
      v2r = v2l;
    } else if (bchi == CAMR_BC_OUTFLOW) {
      qr[ES_RHO] = ql[ES_RHO];
      qr[ES_P] = ql[ES_P];
      qr[ES_REINT] = ql[ES_REINT];
      gamcr = gamcl;
      ur = ul;
      vr = vl;
      v2r = v2l;
    }
  }
  const ROut o =
      (P.riemann_solver == 1)
          ? hllc(ql[ES_RHO], ul, vl, v2l, ql[ES_P], ql[ES_REINT], qr[ES_RHO], ur, vr, v2r,
                 qr[ES_P], qr[ES_REINT], gamcl, gamcr, smallc, P.small_dens, P.small_pres)
          : riemannus(ql[ES_RHO], ul, vl, v2l, ql[ES_P], ql[ES_REINT], qr[ES_RHO], ur, vr, v2r,
                      qr[ES_P], qr[ES_REINT], cav, gamcl, gamcr, P.small, smallc, P.small_dens,
                      P.small_pres, P.smallu);
  constexpr int fu = UMX + dir;
  constexpr int fv = (dir == 0) ? UMY : UMX;
  constexpr int fv2 = (dir == 2) ? UMY : UMZ;
  f[URHO] = o.f_rho;
  f[fu] = o.f_un;
  f[fv] = o.f_ut1;
  f[fv2] = o.f_ut2;
  f[UEDEN] = o.f_eden;
  f[UEINT] = o.f_eint;
  f[UTEMP] = 0.0;
  return o;
}

// Species fluxes of cmpflx (Hydro_cmpflx.H:289-301): the left (ustar > 0),
// right (ustar < 0) or mean (ustar exactly 0, or NaN) species edge states
// times the mass flux, picked by selects.
__device__ __forceinline__ void species_flux(const ROut& o, double* f, const double* ql,
                                             const double* qr) {
  const double flxrho = f[URHO];
  const bool up = o.ustar > 0.0, dn = o.ustar < 0.0;
#pragma unroll
  for (int n = 0; n < NSPEC; ++n) {
    const double a = ql[ES_FS + n], b = qr[ES_FS + n];
    f[UFS + n] = up ? flxrho * a : dn ? flxrho * b : flxrho * 0.50 * (a + b);
  }
}

template <int dir>
__device__ __forceinline__ void cmpflx(double* ql, double* qr, const CellAux& aL,
                                       const CellAux& aR, int idx, int bclo, int bchi,
                                       int domlo, int domhi, const KParams& P, double* f,
                                       double& q_pres, double& q_un) {
  const ROut o = cmpflx_core<dir>(ql, qr, aL, aR, idx, bclo, bchi, domlo, domhi, P, f);
  species_flux(o, f, ql, qr);
  q_pres = o.q_pres;
  q_un = o.q_un;
}

// ---------------------------------------------------------------------------
// PPM (Source/Hydro/Godunov/PPM.H:25-183).
__device__ __forceinline__ void ppm_reconstruct(double s0, double s1, double s2, double s3,
                                                double s4, double flatn, double& sm,
                                                double& sp) {
  double dsl = 2.0 * (s1 - s0);
  double dsr = 2.0 * (s2 - s1);
  double dsvl_l = 0.0;
  if (dsl * dsr > 0.0) {
    const double dsc = 0.5 * (s2 - s0);
    dsvl_l = copysign(1.0, dsc) * dmin(fabs(dsc), dmin(fabs(dsl), fabs(dsr)));
  }
  dsl = 2.0 * (s2 - s1);
  dsr = 2.0 * (s3 - s2);
  double dsvl_r = 0.0;
  if (dsl * dsr > 0.0) {
    const double dsc = 0.5 * (s3 - s1);
    dsvl_r = copysign(1.0, dsc) * dmin(fabs(dsc), dmin(fabs(dsl), fabs(dsr)));
  }
  sm = 0.5 * (s2 + s1) - (1.0 / 6.0) * (dsvl_r - dsvl_l);
  sm = dmax(sm, dmin(s2, s1));
  sm = dmin(sm, dmax(s2, s1));
  // The second pair of van Leer slopes equals the reference's recomputation
  // of the same expressions (PPM.H:63-83): dsvl_l here is dsvl_r above.
  dsvl_l = dsvl_r;
  dsl = 2.0 * (s3 - s2);
  dsr = 2.0 * (s4 - s3);
  dsvl_r = 0.0;
  if (dsl * dsr > 0.0) {
    const double dsc = 0.5 * (s4 - s2);
    dsvl_r = copysign(1.0, dsc) * dmin(fabs(dsc), dmin(fabs(dsl), fabs(dsr)));
  }
  sp = 0.5 * (s3 + s2) - (1.0 / 6.0) * (dsvl_r - dsvl_l);
  sp = dmax(sp, dmin(s3, s2));
  sp = dmin(sp, dmax(s3, s2));
  sm = flatn * sm + (1.0 - flatn) * s2;
  sp = flatn * sp + (1.0 - flatn) * s2;
  if ((sp - s2) * (s2 - sm) <= 0.0) {
    sp = s2;
    sm = s2;
  } else if (fabs(sp - s2) >= 2.0 * fabs(sm - s2)) {
    sp = 3.0 * s2 - 2.0 * sm;
  } else if (fabs(sm - s2) >= 2.0 * fabs(sp - s2)) {
    sm = 3.0 * s2 - 2.0 * sp;
  }
}

// One wave of ppm_int_profile (PPM.H:126-183): the integrals from the right
// (Ip) and left (Im) zone edges for wave speed `speed`.
__device__ __forceinline__ void ppm_wave(double sm, double sp, double s6, double speed,
                                         double dtdx, double& Ip, double& Im) {
  const double sigma = fabs(speed) * dtdx;
  if (speed <= 0.0) {
    Ip = sp;
    Im = sm + 0.5 * sigma * (sp - sm + (1.0 - (2.0 / 3.0) * sigma) * s6);
  } else {
    Ip = sp - 0.5 * sigma * (sp - sm - (1.0 - (2.0 / 3.0) * sigma) * s6);
    Im = sm;
  }
}

// Shock flattening in one direction (Source/Hydro/Godunov/flatten.H:19-99)
// from the pressure p[-3..3] and normal velocity un[-3..3] along it (index
// o+3 holds offset o).  The reference returns 1 when the +-3 stencil leaves
// its q box; every cell traced here has its stencil inside grow(bx,4).
__device__ __forceinline__ double flatten_dir(const double* p, const double* un) {
  const double small_pres = 1.e-200;
  const double shktst = 0.33e0;
  const double zcut1 = 0.75e0;
  const double zcut2 = 0.85e0;
  const double dzcut = 1.0 / (zcut2 - zcut1);
  const double qm = p[2], qp = p[4];
  const double qmun = un[2], qpun = un[4];
  const double qmm = p[1], qpp = p[5];
  double dp = qp - qm;
  const int ishft = (dp > 0.0) ? 1 : -1;
  double denom = dmax(small_pres, fabs(qpp - qmm));
  double zeta = fabs(dp) / denom;
  const double z = dmin(1.0, dmax(0.0, dzcut * (zeta - zcut1)));
  double tst = (qmun - qpun >= 0.0) ? 1.0 : 0.0;
  double tmp = dmin(qp, qm);
  const double chi = (fabs(dp) / tmp) > shktst ? tst : 0.0;
  // offsets 1-ishft, -(1+ishft), 2-ishft, -(2+ishft) (flatten.H:78-83),
  // with ishft = +-1 spelled out so the stencil stays in registers
  const bool up = ishft == 1;
  const double qpshft = up ? p[3] : p[5];
  const double qmshft = up ? p[1] : p[3];
  const double qpunshft = up ? un[3] : un[5];
  const double qmunshft = up ? un[1] : un[3];
  const double qppshft = up ? p[4] : p[6];
  const double qmmshft = up ? p[0] : p[2];
  dp = qpshft - qmshft;
  denom = dmax(small_pres, fabs(qppshft - qmmshft));
  zeta = fabs(dp) / denom;
  const double z2 = dmin(1.0, dmax(0.0, dzcut * (zeta - zcut1)));
  tst = (qmunshft - qpunshft >= 0.0) ? 1.0 : 0.0;
  tmp = dmin(qpshft, qmshft);
  const double chi2 = (fabs(dp) / tmp) > shktst ? tst : 0.0;
  return 1.0 - dmax(chi2 * z2, chi * z);
}

// Characteristic projection of PPM.cpp:204-310 (plus state, side = +1 uses
// the "Im" integrals and the left-moving waves) and :313-409 (minus state).
// ref[w] are the integrals of rho, un, p, rhoe for waves w = 0 (u-c), 1 (u),
// 2 (u+c) toward the face; gam_ref the traced gamma.
struct Traced4 {
  double rho[3], un[3], p[3], re[3];
};

__device__ __forceinline__ void ppm_project(const Traced4& I, int wref, double gam_ref,
                                            double un, double cc, bool plus_state,
                                            const KParams& P, double& o_rho, double& o_un,
                                            double& o_p, double& o_re) {
  double rho_ref = I.rho[wref];
  const double un_ref = I.un[wref];
  double p_ref = I.p[wref];
  const double rhoe_g_ref = I.re[wref];
  rho_ref = dmax(rho_ref, P.small_dens);
  const double rho_ref_inv = 1.0 / rho_ref;
  p_ref = dmax(p_ref, P.small_pres);
  const double cc_ref = sqrt(gam_ref * p_ref / rho_ref);
  const double csq_ref = cc_ref * cc_ref;
  const double cc_ref_inv = 1.0 / cc_ref;
  const double h_g_ref = (p_ref + rhoe_g_ref) * rho_ref_inv / csq_ref;
  const double dum = un_ref - I.un[0];
  const double dptotm = p_ref - I.p[0];
  const double drho = rho_ref - I.rho[1];
  const double dptot = p_ref - I.p[1];
  const double drhoe_g = rhoe_g_ref - I.re[1];
  const double dup = un_ref - I.un[2];
  const double dptotp = p_ref - I.p[2];
  double alpham = 0.5 * (dptotm * rho_ref_inv * cc_ref_inv - dum) * rho_ref * cc_ref_inv;
  double alphap = 0.5 * (dptotp * rho_ref_inv * cc_ref_inv + dup) * rho_ref * cc_ref_inv;
  double alpha0r = drho - dptot / csq_ref;
  double alpha0e_g = drhoe_g - dptot * h_g_ref;
  if (plus_state) {
    if (un - cc > 0.) alpham = 0.;
    else if (un - cc < 0.) alpham *= -1.0;
    else alpham *= -0.5;
    if (un + cc > 0.) alphap = 0.;
    else if (un + cc < 0.) alphap *= -1.0;
    else alphap *= -0.5;
    if (un > 0.) { alpha0r = 0.; alpha0e_g = 0.; }
    else if (un < 0.) { alpha0r *= -1.0; alpha0e_g *= -1.0; }
    else { alpha0r *= -0.5; alpha0e_g *= -0.5; }
  } else {
    if (un - cc > 0.) alpham *= -1.0;
    else if (un - cc < 0.) alpham = 0.;
    else alpham *= -0.5;
    if (un + cc > 0.) alphap *= -1.0;
    else if (un + cc < 0.) alphap = 0.;
    else alphap *= -0.5;
    if (un > 0.) { alpha0r *= -1.0; alpha0e_g *= -1.0; }
    else if (un < 0.) { alpha0r = 0.; alpha0e_g = 0.; }
    else { alpha0r *= -0.5; alpha0e_g *= -0.5; }
  }
  o_rho = rho_ref + alphap + alpham + alpha0r;
  o_un = un_ref + (alphap - alpham) * cc_ref * rho_ref_inv;
  o_p = p_ref + (alphap + alpham) * csq_ref;
  o_rho = dmax(o_rho, P.small_dens);
  // The minus state's pressure is floored with small_dens in the reference
  // (PPM.cpp:398); the plus state's with small_pres (:295).
  o_p = dmax(o_p, plus_state ? P.small_pres : P.small_dens);
  o_re = rhoe_g_ref + (alphap + alpham) * h_g_ref * csq_ref + alpha0e_g;
}

// ---------------------------------------------------------------------------
// PLM slope (Source/Hydro/Godunov/PLM.H:19-79) from q at offsets -2..2.
__device__ __forceinline__ double plm_slope(double qm2, double qm, double qc, double qp,
                                            double qp2, double flat, int order) {
  if (order == 1) return 0.;
  double dlft, drgt, dcen, dfm = 0.0, dfp = 0.0, dlim, dsgn, dtemp;
  if (order == 4) {
    dlft = qm - qm2;
    drgt = qc - qm;
    dcen = 0.5 * (dlft + drgt);
    dsgn = copysign(1.0, dcen);
    dlim = (dlft * drgt >= 0.0) ? 2.0 * dmin(fabs(dlft), fabs(drgt)) : 0.0;
    dfm = dsgn * dmin(dlim, fabs(dcen));
    dlft = qp - qc;
    drgt = qp2 - qp;
    dcen = 0.5 * (dlft + drgt);
    dsgn = copysign(1.0, dcen);
    dlim = (dlft * drgt >= 0.0) ? 2.0 * dmin(fabs(dlft), fabs(drgt)) : 0.0;
    dfp = dsgn * dmin(dlim, fabs(dcen));
  }
  dlft = qc - qm;
  drgt = qp - qc;
  dcen = 0.5 * (dlft + drgt);
  dsgn = copysign(1.0, dcen);
  dlim = (dlft * drgt >= 0.0) ? 2.0 * dmin(fabs(dlft), fabs(drgt)) : 0.0;
  dtemp = 4.0 / 3.0 * dcen - 1.0 / 6.0 * (dfp + dfm);
  return flat * dsgn * dmin(dlim, fabs(dtemp));
}

// plm_pslope (Source/Hydro/Godunov/PLM.H:84-165): the pressure slope with
// the hydrostatic part rho * src_u * dx taken out of each difference and
// added back at the end (use_pslope = 1).  p, r, su: the 5-point stencils
// of pressure, density and the primitive source of the normal velocity.
__device__ __forceinline__ double plm_pslope(const double* p, const double* r, const double* su,
                                             double dx, double flat, int order) {
  if (order == 1) return 0.;
  double dlft, drgt, dcen, dfm = 0.0, dfp = 0.0, dlim, dsgn, dtemp;
  const double qm2 = p[0], qm = p[1], qc = p[2], qp = p[3], qp2 = p[4];
  if (order == 4) {
    dlft = qm - qm2 - 0.25 * dx * (r[1] + r[0]) * (su[1] + su[0]);
    drgt = qc - qm - 0.25 * dx * (r[1] + r[2]) * (su[1] + su[2]);
    dcen = 0.5 * (dlft + drgt);
    dsgn = copysign(1.0, dcen);
    dlim = (dlft * drgt >= 0.0) ? 2.0 * dmin(fabs(dlft), fabs(drgt)) : 0.0;
    dfm = dsgn * dmin(dlim, fabs(dcen));
    dlft = qp - qc - 0.25 * dx * (r[3] + r[2]) * (su[3] + su[2]);
    drgt = qp2 - qp - 0.25 * dx * (r[3] + r[4]) * (su[3] + su[4]);
    dcen = 0.5 * (dlft + drgt);
    dsgn = copysign(1.0, dcen);
    dlim = (dlft * drgt >= 0.0) ? 2.0 * dmin(fabs(dlft), fabs(drgt)) : 0.0;
    dfp = dsgn * dmin(dlim, fabs(dcen));
  }
  dlft = qc - qm - 0.25 * dx * (r[2] + r[1]) * (su[2] + su[1]);
  drgt = qp - qc - 0.25 * dx * (r[2] + r[3]) * (su[2] + su[3]);
  dcen = 0.5 * (dlft + drgt);
  dsgn = copysign(1.0, dcen);
  dlim = (dlft * drgt >= 0.0) ? 2.0 * dmin(fabs(dlft), fabs(drgt)) : 0.0;
  dtemp = 4.0 / 3.0 * dcen - 1.0 / 6.0 * (dfp + dfm);
  double dp = flat * dsgn * dmin(dlim, fabs(dtemp));
  dp += r[2] * su[2] * dx;
  return dp;
}

// ---------------------------------------------------------------------------
// Transverse corrections (Source/Hydro/Godunov/Godunov_utils_3D.H).  The
// reference's transdo/transdd each fill the plus state on a cell's low face
// and the minus state on its high face from shared flux differences; here a
// face thread evaluates the half it needs of each of its two cells.
struct TTerms {
  double flxrho, flxu, flxv, flxw, flxe;
  double compn[NSPEC];
  double dAup, pav, dAu;
};

// hydro_transdo :74-122, from the E-flux records on the cell's low/high
// E-faces (FR_* layout).
__device__ __forceinline__ TTerms transdo_terms(const double* lo, const double* hi,
                                                double cdtdx) {
  TTerms t;
  t.flxrho = cdtdx * (hi[FR_RHO] - lo[FR_RHO]);
  t.flxu = cdtdx * (hi[FR_MX] - lo[FR_MX]);
  t.flxv = cdtdx * (hi[FR_MY] - lo[FR_MY]);
  t.flxw = cdtdx * (hi[FR_MZ] - lo[FR_MZ]);
  t.flxe = cdtdx * (hi[FR_E] - lo[FR_E]);
#pragma unroll
  for (int s = 0; s < NSPEC; ++s) t.compn[s] = cdtdx * (hi[FR_FS + s] - lo[FR_FS + s]);
  const double pggp = hi[FR_PRES];
  const double pggm = lo[FR_PRES];
  const double ugp = hi[FR_UN];
  const double ugm = lo[FR_UN];
  t.dAup = pggp * ugp - pggm * ugm;
  t.pav = 0.5 * (pggp + pggm);
  t.dAu = ugp - ugm;
  return t;
}

// One side of hydro_transdo (:82-238).
__device__ __forceinline__ void transdo_side(const TTerms& t, double c, const double* qn,
                                             double cdtdx, const KParams& P, double* out) {
#pragma unroll
  for (int s = 0; s < NSPEC; ++s) {
    const double rr = qn[ES_RHO];
    const double rrnew = rr - t.flxrho;
    const double compo = rr * qn[ES_FS + s] - t.compn[s];
    out[ES_FS + s] = compo / rrnew;
  }
  const double rrr = qn[ES_RHO];
  double rur = qn[ES_U];
  double rvr = qn[ES_V];
  double rwr = qn[ES_W];
  const double ekinr = 0.5 * rrr * (rur * rur + rvr * rvr + rwr * rwr);
  rur *= rrr;
  rvr *= rrr;
  rwr *= rrr;
  const double rer = qn[ES_REINT] + ekinr;
  double rrnewr = rrr - t.flxrho;
  double runewr = rur - t.flxu;
  double rvnewr = rvr - t.flxv;
  double rwnewr = rwr - t.flxw;
  double renewr = rer - t.flxe;
  bool reset_state = false;
  if (P.transverse_reset_density == 1 && rrnewr < 0.) {
    rrnewr = rrr;
    runewr = rur;
    rvnewr = rvr;
    rwnewr = rwr;
    renewr = rer;
    reset_state = true;
  }
  out[ES_RHO] = rrnewr;
  out[ES_U] = runewr / rrnewr;
  out[ES_V] = rvnewr / rrnewr;
  out[ES_W] = rwnewr / rrnewr;
  const double rhoekinr = 0.5 * (runewr * runewr + rvnewr * rvnewr + rwnewr * rwnewr) / rrnewr;
  out[ES_REINT] = renewr - rhoekinr;
  if (!reset_state) {
    const double pnewr = qn[ES_P] - cdtdx * (t.dAup + t.pav * t.dAu * (c - 1.0));
    out[ES_P] = dmax(pnewr, P.small_pres);
  } else {
    out[ES_P] = qn[ES_P];
  }
}

struct TDTerms {
  double flxrho, flxu, flxv, flxw, flxe;
  double compn[NSPEC];
  double pxnew, pynew;
};

// hydro_transdd :307-384 from the t0-face records (f0) and t1-face records (f1).
__device__ __forceinline__ TDTerms transdd_terms(const double* f0lo, const double* f0hi,
                                                 const double* f1lo, const double* f1hi,
                                                 double c, double cdtdx0, double cdtdx1) {
  TDTerms t;
  t.flxrho = cdtdx0 * (f0hi[FR_RHO] - f0lo[FR_RHO]) + cdtdx1 * (f1hi[FR_RHO] - f1lo[FR_RHO]);
  t.flxu = cdtdx0 * (f0hi[FR_MX] - f0lo[FR_MX]) + cdtdx1 * (f1hi[FR_MX] - f1lo[FR_MX]);
  t.flxv = cdtdx0 * (f0hi[FR_MY] - f0lo[FR_MY]) + cdtdx1 * (f1hi[FR_MY] - f1lo[FR_MY]);
  t.flxw = cdtdx0 * (f0hi[FR_MZ] - f0lo[FR_MZ]) + cdtdx1 * (f1hi[FR_MZ] - f1lo[FR_MZ]);
  t.flxe = cdtdx0 * (f0hi[FR_E] - f0lo[FR_E]) + cdtdx1 * (f1hi[FR_E] - f1lo[FR_E]);
#pragma unroll
  for (int s = 0; s < NSPEC; ++s) {
    t.compn[s] = cdtdx0 * (f0hi[FR_FS + s] - f0lo[FR_FS + s]) +
                 cdtdx1 * (f1hi[FR_FS + s] - f1lo[FR_FS + s]);
  }
  const double pggpx = f0hi[FR_PRES];
  const double pggmx = f0lo[FR_PRES];
  const double ugpx = f0hi[FR_UN];
  const double ugmx = f0lo[FR_UN];
  const double dAupx = pggpx * ugpx - pggmx * ugmx;
  const double pavx = 0.5 * (pggpx + pggmx);
  const double dAux = ugpx - ugmx;
  const double pggpy = f1hi[FR_PRES];
  const double pggmy = f1lo[FR_PRES];
  const double ugpy = f1hi[FR_UN];
  const double ugmy = f1lo[FR_UN];
  const double dAupy = pggpy * ugpy - pggmy * ugmy;
  const double pavy = 0.5 * (pggpy + pggmy);
  const double dAuy = ugpy - ugmy;
  t.pxnew = cdtdx0 * (dAupx + pavx * dAux * (c - 1.0));
  t.pynew = cdtdx1 * (dAupy + pavy * dAuy * (c - 1.0));
  return t;
}

// One side of hydro_transdd (:326-481).  srcq: primitive sources of the cell
// in ES_* order (all +0 for zero sources).
__device__ __forceinline__ void transdd_side(const TDTerms& t, const double* qn,
                                             const double* srcq, double hdt,
                                             const KParams& P, double* out) {
  const double rrr = qn[ES_RHO];
  double rrnewr = rrr - t.flxrho;
#pragma unroll
  for (int s = 0; s < NSPEC; ++s) {
    const double compo = rrr * qn[ES_FS + s] - t.compn[s];
    out[ES_FS + s] = compo / rrnewr + hdt * srcq[ES_FS + s];
  }
  const double rur = rrr * qn[ES_U];
  const double rvr = rrr * qn[ES_V];
  const double rwr = rrr * qn[ES_W];
  const double ekinr = 0.5 * (rur * rur + rvr * rvr + rwr * rwr) / rrr;
  const double rer = qn[ES_REINT] + ekinr;
  double runewr = rur - t.flxu;
  double rvnewr = rvr - t.flxv;
  double rwnewr = rwr - t.flxw;
  double renewr = rer - t.flxe;
  bool reset_state = false;
  if (P.transverse_reset_density == 1 && rrnewr < 0.) {
    rrnewr = rrr;
    runewr = rur;
    rvnewr = rvr;
    rwnewr = rwr;
    renewr = rer;
    reset_state = true;
  }
  out[ES_RHO] = rrnewr + hdt * srcq[ES_RHO];
  out[ES_U] = runewr / rrnewr + hdt * srcq[ES_U];
  out[ES_V] = rvnewr / rrnewr + hdt * srcq[ES_V];
  out[ES_W] = rwnewr / rrnewr + hdt * srcq[ES_W];
  const double rhoekinr = 0.5 * (runewr * runewr + rvnewr * rvnewr + rwnewr * rwnewr) / rrnewr;
  out[ES_REINT] = renewr - rhoekinr + hdt * srcq[ES_REINT];
  double pout;
  if (!reset_state) {
    pout = qn[ES_P] - t.pxnew - t.pynew + hdt * srcq[ES_P];
  } else {
    pout = qn[ES_P] + hdt * srcq[ES_P];
  }
  out[ES_P] = dmax(pout, P.small_pres);
}

// ---------------------------------------------------------------------------
// MOL limiter (Source/Hydro/MOL/MOL_hydro_K.H:11-20).
__device__ __forceinline__ double mol_limiter(double dlft, double drgt, double plm_theta) {
  const double dcen = 0.5 * (dlft + drgt);
  const double dsgn = copysign(1.0, dcen);
  const double slop = plm_theta * dmin(fabs(dlft), fabs(drgt));
  const double dlim = (dlft * drgt >= 0.0) ? slop : 0.0;
  return dsgn * dmin(dlim, fabs(dcen));
}

// EOS pieces (Source/EOS/GammaLaw/EOS.H): T from e, E from T.
__device__ __forceinline__ double eos_ey2t(double gamma, double e) {
  const double poverrho = (gamma - 1.0) * e;
  return poverrho * AIRMW / RU;
}

__device__ __forceinline__ double eos_rty2e(double gamma, double t, const double* y) {
  const double cv = RU / (AIRMW * (gamma - 1.0));
  double e = 0.0;
#pragma unroll
  for (int n = 0; n < NSPEC; ++n) e += y[n] * (cv * t);
  return e;
}

}  // namespace camr
