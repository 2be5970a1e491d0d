// Per-cell and per-face device bodies shared by the box hydro kernels
// (hydro_kernels.cu) and the embedded-boundary kernels (eb.cu).  Each one
// reproduces the reference's arithmetic operation by operation.
#pragma once

#include "hydro_point.cuh"
#include "rndiv.h"


namespace camr {

// Loads of arrays that a kernel only reads go through the read-only data
// path when CAMR_LDG is 1 (the default).
#ifndef CAMR_LDG
#define CAMR_LDG 1
#endif
__device__ __forceinline__ double ld_ro(const double* p) {
#if CAMR_LDG
  return __ldg(p);
#else
  return *p;
#endif
}

__device__ __forceinline__ void load_es(const double* a, const Space& s, int64_t at, double* r) {
#pragma unroll
  for (int n = 0; n < ES_N; ++n) r[n] = ld_ro(a + at + n * s.sn);
}
__device__ __forceinline__ void store_es(double* a, const Space& s, int64_t at, const double* r) {
#pragma unroll
  for (int n = 0; n < ES_N; ++n) a[at + n * s.sn] = r[n];
}
__device__ __forceinline__ void load_fr(const double* a, const Space& s, int64_t at, double* r) {
#pragma unroll
  for (int n = 0; n < FR_N; ++n) r[n] = ld_ro(a + at + n * s.sn);
}
__device__ __forceinline__ CellAux load_aux(const double* q, const Space& s, int64_t at,
                                            double gamma) {
  CellAux a;
  a.c = ld_ro(q + at + SQ_C * s.sn);
  a.csml = ld_ro(q + at + SQ_CSML * s.sn);
  a.gamc = gamma;  // qaux QGAMC = EOS::REY2Gam = gamma (Hydro_ctoprim.H:83,96)
  return a;
}

// ---------------------------------------------------------------------------
// K1: conservative -> primitive (Source/Hydro/Hydro_ctoprim.H:11-101) and,
// with sources, primitive sources (:106-157).
__device__ __forceinline__ void ctoprim_body(int i, int j, int k, const Space& s, const DFab& u,
                                             const DFab& src, bool has_src, const KParams& P,
                                             double* q, double* srcq, DevError* err) {
  const int64_t at = s.idx(i, j, k);
  const double rho = u(i, j, k, URHO);
  if (!(rho > 0.)) {
    // The reference leaves q untouched here; downstream use is undefined.
    report_error(err, 1, i, j, k);
    return;
  }
  const double rhoinv = 1.0 / rho;
  const double vx = u(i, j, k, UMX) * rhoinv;
  const double vy = u(i, j, k, UMY) * rhoinv;
  const double vz = u(i, j, k, UMZ) * rhoinv;
  const double kineng = 0.5 * rho * (vx * vx + vy * vy + vz * vz);
  const double ueden = u(i, j, k, UEDEN);
  const double ueint = u(i, j, k, UEINT);
  if (!P.allow_negative_energy && (!(ueden > 0.) || !(ueint > 0.))) report_error(err, 1, i, j, k);
  double e;
  if ((ueden - kineng) / ueden > P.dual_energy_eta1) {
    e = (ueden - kineng) * rhoinv;
  } else {
    e = ueint * rhoinv;
  }
  double y[NSPEC];
#pragma unroll
  for (int sp = 0; sp < NSPEC; ++sp) y[sp] = u(i, j, k, UFS + sp) * rhoinv;
  const double p = (P.gamma - 1.0) * rho * e;
  const double rhoe = e * rho;
  const double cs = sqrt(P.gamma * p / rho);
  q[at + SQ_RHO * s.sn] = rho;
  q[at + SQ_U * s.sn] = vx;
  q[at + SQ_V * s.sn] = vy;
  q[at + SQ_W * s.sn] = vz;
  q[at + SQ_P * s.sn] = p;
  q[at + SQ_REINT * s.sn] = rhoe;
#pragma unroll
  for (int sp = 0; sp < NSPEC; ++sp) q[at + (SQ_FS + sp) * s.sn] = y[sp];
  q[at + SQ_C * s.sn] = cs;
  q[at + SQ_CSML * s.sn] = dmax(P.small_num, P.small_num * cs);
  if (has_src) {
    // hydro_srctoprim with the EOS derivatives of ctoprim
    // (QDPDE = (gamma-1)*rho, QDPDR = (gamma-1)*e).
    const double dpde = (P.gamma - 1.0) * rho;
    const double dpdr = (P.gamma - 1.0) * e;
    const double srcrho = src(i, j, k, URHO);
    const double sq_reint = src(i, j, k, UEINT);
    srcq[at + ES_RHO * s.sn] = srcrho;
    srcq[at + ES_U * s.sn] = (src(i, j, k, UMX) - vx * srcrho) * rhoinv;
    srcq[at + ES_V * s.sn] = (src(i, j, k, UMY) - vy * srcrho) * rhoinv;
    srcq[at + ES_W * s.sn] = (src(i, j, k, UMZ) - vz * srcrho) * rhoinv;
    srcq[at + ES_REINT * s.sn] = sq_reint;
#pragma unroll
    for (int sp = 0; sp < NSPEC; ++sp) {
      srcq[at + (ES_FS + sp) * s.sn] = (src(i, j, k, UFS + sp) - y[sp] * srcrho) * rhoinv;
    }
    srcq[at + ES_P * s.sn] = dpde * (sq_reint - rhoe * srcrho * rhoinv) * rhoinv + dpdr * srcrho;
  }
}


// ---------------------------------------------------------------------------
// MOL slopes (Source/Hydro/MOL/MOL_hydro_K.H:24-255) of a cell in direction
// blockIdx.y.  Slot 1 (entropy) is never read by mol_riemann_{x,y,z} and is
// not produced.  Stored slots: 0, 2, 3, 4, QREINT, species.
enum { SL_0 = 0, SL_2 = 1, SL_3 = 2, SL_4 = 3, SL_RE = 4, SL_FS = 5, SL_N = 8 };

// hydro_plm_d (Godunov/PLM.H:170-323) of one cell in direction d from its
// slopes (ES_N slots): the plus state on the cell's low face (qp_o) and the
// minus state on its high face (qm_o).
template <int d>
__device__ __forceinline__ void plm_edge_states(const double* q, int64_t at, int64_t sn,
                                                const double* slope, double dtdx,
                                                const KParams& P, double* qp_o,
                                                double* qm_o) {
  constexpr int l0 = d;
  constexpr int l1 = (d == 0) ? 1 : 0;
  constexpr int l2 = (d == 2) ? 1 : 2;
  const double cc = ld_ro(q + at + SQ_C * sn);
  const double dtdx_p = dtdx;
  const double cs = cc * cc;
  const double rho = ld_ro(q + at + SQ_RHO * sn);
  const double vel[3] = {ld_ro(q + at + SQ_U * sn), ld_ro(q + at + SQ_V * sn),
                         ld_ro(q + at + SQ_W * sn)};
  const double pr = ld_ro(q + at + SQ_P * sn);
  const double rhoe = ld_ro(q + at + SQ_REINT * sn);
  const double enth = ((rhoe + pr) / rho) / cs;
  const double drho = slope[ES_RHO];
  const double dvel[3] = {slope[ES_U], slope[ES_V], slope[ES_W]};
  const double dp = slope[ES_P];
  const double drhoe = slope[ES_REINT];
  const double alpham = 0.5 * (dp / (rho * cc) - dvel[d]) * rho / cc;
  const double alphap = 0.5 * (dp / (rho * cc) + dvel[d]) * rho / cc;
  const double alpha0r = drho - dp / cs;
  const double alpha0e = drhoe - dp * enth;
  const double alpha0v = dvel[l1];
  const double alpha0w = dvel[l2];
  const double wv[3] = {vel[d] - cc, vel[d], vel[d] + cc};
  {
    const double rho_ref = rho - 0.5 * (1.0 + dtdx_p * dmin(wv[0], 0.0)) * drho;
    double vel_ref[3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
      vel_ref[a] = vel[a] - 0.5 * (1.0 + dtdx_p * dmin(wv[0], 0.0)) * dvel[a];
    const double p_ref = pr - 0.5 * (1.0 + dtdx_p * dmin(wv[0], 0.0)) * dp;
    const double rhoe_ref = rhoe - 0.5 * (1.0 + dtdx_p * dmin(wv[0], 0.0)) * drhoe;
    const double apright = 0.25 * dtdx_p * (wv[0] - wv[2]) * (1.0 - copysign(1.0, wv[2])) * alphap;
    const double amright = 0.0;
    const double azrright = 0.25 * dtdx_p * (wv[0] - wv[1]) * (1.0 - copysign(1.0, wv[1])) * alpha0r;
    const double azeright = 0.25 * dtdx_p * (wv[0] - wv[1]) * (1.0 - copysign(1.0, wv[1])) * alpha0e;
    const double azv1rght = 0.25 * dtdx_p * (wv[0] - wv[1]) * (1.0 - copysign(1.0, wv[1])) * alpha0v;
    const double azw1rght = 0.25 * dtdx_p * (wv[0] - wv[1]) * (1.0 - copysign(1.0, wv[1])) * alpha0w;
    double r0 = rho_ref + apright + amright + azrright;
    qp_o[ES_RHO] = dmax(r0, P.small_dens);
    qp_o[ES_U + l0] = vel_ref[l0] + (apright - amright) * cc / rho;
    qp_o[ES_U + l1] = vel_ref[l1] + azv1rght;
    qp_o[ES_U + l2] = vel_ref[l2] + azw1rght;
    double p0 = p_ref + (apright + amright) * cs;
    qp_o[ES_P] = dmax(p0, P.small_pres);
    qp_o[ES_REINT] = rhoe_ref + (apright + amright) * enth * cs + azeright;
  }
  {
    const double rho_ref = rho + 0.5 * (1.0 - dtdx_p * dmax(wv[2], 0.0)) * drho;
    double vel_ref[3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
      vel_ref[a] = vel[a] + 0.5 * (1.0 - dtdx_p * dmax(wv[2], 0.0)) * dvel[a];
    const double p_ref = pr + 0.5 * (1.0 - dtdx_p * dmax(wv[2], 0.0)) * dp;
    const double rhoe_ref = rhoe + 0.5 * (1.0 - dtdx_p * dmax(wv[2], 0.0)) * drhoe;
    const double apleft = 0.0;
    const double amleft = 0.25 * dtdx_p * (wv[2] - wv[0]) * (1.0 + copysign(1.0, wv[0])) * alpham;
    const double azrleft = 0.25 * dtdx_p * (wv[2] - wv[1]) * (1.0 + copysign(1.0, wv[1])) * alpha0r;
    const double azeleft = 0.25 * dtdx_p * (wv[2] - wv[1]) * (1.0 + copysign(1.0, wv[1])) * alpha0e;
    const double azv1left = 0.25 * dtdx_p * (wv[2] - wv[1]) * (1.0 + copysign(1.0, wv[1])) * alpha0v;
    const double azw1left = 0.25 * dtdx_p * (wv[2] - wv[1]) * (1.0 + copysign(1.0, wv[1])) * alpha0w;
    double r0 = rho_ref + apleft + amleft + azrleft;
    qm_o[ES_RHO] = dmax(r0, P.small_dens);
    qm_o[ES_U + l0] = vel_ref[l0] + (apleft - amleft) * cc / rho;
    qm_o[ES_U + l1] = vel_ref[l1] + azv1left;
    qm_o[ES_U + l2] = vel_ref[l2] + azw1left;
    double p0 = p_ref + (apleft + amleft) * cs;
    qm_o[ES_P] = dmax(p0, P.small_pres);
    qm_o[ES_REINT] = rhoe_ref + (apleft + amleft) * enth * cs + azeleft;
  }
  const double vel_ad = vel[l0];
#pragma unroll
  for (int sp = 0; sp < NSPEC; ++sp) {
    const double qn = ld_ro(q + at + (SQ_FS + sp) * sn);
    {
      const double spzero = (vel_ad > 0) ? -1.0 : vel_ad * dtdx_p;
      const double acmprght = 0.5 * (-1.0 - spzero) * slope[ES_FS + sp];
      qp_o[ES_FS + sp] = qn + acmprght;
    }
    {
      const double spzero = vel_ad >= 0 ? vel_ad * dtdx_p : 1.0;
      const double acmpleft = 0.5 * (1.0 - spzero) * slope[ES_FS + sp];
      qm_o[ES_FS + sp] = qn + acmpleft;
    }
  }}

template <int d>
__device__ __forceinline__ void mol_slope_compute(int64_t at, const Space& s, const KParams& P,
                                                  const double* q, double* o) {
  const int64_t st = (d == 0) ? 1 : (d == 1) ? s.sy : s.sz;
  if (P.plm_iorder == 1) {
#pragma unroll
    for (int n = 0; n < SL_N; ++n) o[n] = 0.;
    return;
  }
  const double plm_theta = 2.0;
  auto Q = [&](int off, int slot) { return ld_ro(q + at + off * st + slot * s.sn); };
  constexpr int un = SQ_U + d;
  constexpr int t1 = (d == 0) ? SQ_V : SQ_U;
  constexpr int t2 = (d == 2) ? SQ_V : SQ_W;
  const double c = Q(0, SQ_C);
  const double cs2 = c * c;
  const double dpl = Q(0, SQ_P) - Q(-1, SQ_P);
  const double dpr = Q(1, SQ_P) - Q(0, SQ_P);
  const double enth = (Q(0, SQ_REINT) + Q(0, SQ_P)) / dmax(Q(0, SQ_RHO), P.small_dens);
  // the reference's quotients by c (2) and by c^2 (8); with every operand
  // in range they come from the two reciprocals (rn_div_unchecked, the
  // same bits as the divisions), else from the divisions
  const double nc[2] = {0.5 * dpl, 0.5 * dpr};
  double ns[2 + 2 * NSPEC];
  ns[0] = enth * dpl;
  ns[1] = enth * dpr;
#pragma unroll
  for (int sp = 0; sp < NSPEC; ++sp) {
    ns[2 + 2 * sp] = Q(0, SQ_FS + sp) * dpl;
    ns[3 + 2 * sp] = Q(0, SQ_FS + sp) * dpr;
  }
  bool ok = rd_in_range(c) & rd_in_range(cs2) & rd_in_range(nc[0]) & rd_in_range(nc[1]);
#pragma unroll
  for (int m = 0; m < 2 + 2 * NSPEC; ++m) ok = ok & rd_in_range(ns[m]);
  double qc[2], qs[2 + 2 * NSPEC];
  if (ok) {
    const double ic = 1.0 / c, ics2 = 1.0 / cs2;
#pragma unroll
    for (int m = 0; m < 2; ++m) qc[m] = rn_div_unchecked(nc[m], c, ic);
#pragma unroll
    for (int m = 0; m < 2 + 2 * NSPEC; ++m) qs[m] = rn_div_unchecked(ns[m], cs2, ics2);
  } else {
#pragma unroll
    for (int m = 0; m < 2; ++m) qc[m] = nc[m] / c;
#pragma unroll
    for (int m = 0; m < 2 + 2 * NSPEC; ++m) qs[m] = ns[m] / cs2;
  }
  double dlft = qc[0] - 0.5 * Q(0, SQ_RHO) * (Q(0, un) - Q(-1, un));
  double drgt = qc[1] - 0.5 * Q(0, SQ_RHO) * (Q(1, un) - Q(0, un));
  o[SL_0] = mol_limiter(dlft, drgt, plm_theta);
  dlft = qc[0] + 0.5 * Q(0, SQ_RHO) * (Q(0, un) - Q(-1, un));
  drgt = qc[1] + 0.5 * Q(0, SQ_RHO) * (Q(1, un) - Q(0, un));
  o[SL_2] = mol_limiter(dlft, drgt, plm_theta);
  dlft = Q(0, t1) - Q(-1, t1);
  drgt = Q(1, t1) - Q(0, t1);
  o[SL_3] = mol_limiter(dlft, drgt, plm_theta);
  dlft = Q(0, t2) - Q(-1, t2);
  drgt = Q(1, t2) - Q(0, t2);
  o[SL_4] = mol_limiter(dlft, drgt, plm_theta);
  dlft = (Q(0, SQ_REINT) - Q(-1, SQ_REINT)) - qs[0];
  drgt = (Q(1, SQ_REINT) - Q(0, SQ_REINT)) - qs[1];
  o[SL_RE] = mol_limiter(dlft, drgt, plm_theta);
#pragma unroll
  for (int sp = 0; sp < NSPEC; ++sp) {
    const int n = SQ_FS + sp;
    dlft = Q(0, SQ_RHO) * Q(0, n) - Q(-1, SQ_RHO) * Q(-1, n) - qs[2 + 2 * sp];
    drgt = Q(1, SQ_RHO) * Q(1, n) - Q(0, SQ_RHO) * Q(0, n) - qs[3 + 2 * sp];
    o[SL_FS + sp] = mol_limiter(dlft, drgt, plm_theta);
  }
}

template <int d>
__device__ __forceinline__ void mol_slope_body(int i, int j, int k, const Space& s,
                                               const KParams& P, const double* q, double* o) {
  const int64_t at = s.idx(i, j, k);
  double sl[SL_N];
  mol_slope_compute<d>(at, s, P, q, sl);
#pragma unroll
  for (int n = 0; n < SL_N; ++n) o[at + n * s.sn] = sl[n];
}

// MOL face of direction d at (i,j,k) (between the cells at -e_d and 0): the
// edge states of mol_riemann_{x,y,z} (MOL_riemann_K.H:12-488) and
// hydro_cmpflx's Riemann flux (Hydro_cmpflx.H:153-311), before
// adjust_fluxes.
template <int d>
__device__ __forceinline__ void mol_edges_cmpflx(int i, int j, int k, const Space& s,
                                                 const KGeom& g, const KParams& P,
                                                 const double* q, const double* sl, double* f,
                                                 double& qpres, double& qun) {
  const int64_t at = s.idx(i, j, k);
  const int64_t st = (d == 0) ? 1 : (d == 1) ? s.sy : s.sz;
  const int64_t atL = at - st;
  auto Q = [&](int64_t c, int slot) { return ld_ro(q + c + slot * s.sn); };
  auto S = [&](int64_t c, int slot) { return ld_ro(sl + c + slot * s.sn); };
  constexpr int un = SQ_U + d;
  constexpr int t1 = (d == 0) ? SQ_V : SQ_U;
  constexpr int t2 = (d == 2) ? SQ_V : SQ_W;
  double ql[ES_N], qr[ES_N];
  {
    const double cspeed = Q(atL, SQ_C);
    const double enth = (Q(atL, SQ_REINT) + Q(atL, SQ_P)) / dmax(Q(atL, SQ_RHO), P.small_dens);
    const double d0 = S(atL, SL_0), d2 = S(atL, SL_2);
    double pl = Q(atL, SQ_P) + 0.5 * (d0 + d2) * cspeed;
    ql[ES_P] = dmax(pl, P.small_pres);
    ql[ES_U + d] = Q(atL, un) + 0.5 * ((d2 - d0) / Q(atL, SQ_RHO));
    ql[ES_U + (t1 - SQ_U)] = Q(atL, t1) + 0.5 * S(atL, SL_3);
    ql[ES_U + (t2 - SQ_U)] = Q(atL, t2) + 0.5 * S(atL, SL_4);
    // the four quotients by cspeed, then the three by sum, each group from
    // one reciprocal (rn_div_group: the same bits as the divisions)
    double nq[NSPEC + 1], qq[NSPEC + 1];
#pragma unroll
    for (int sp = 0; sp < NSPEC; ++sp) nq[sp] = Q(atL, SQ_FS + sp) * (d0 + d2);
    nq[NSPEC] = enth * (d0 + d2);
    rn_div_group<NSPEC + 1>(nq, cspeed, qq);
    double sum = 0.;
#pragma unroll
    for (int sp = 0; sp < NSPEC; ++sp) {
      const double specden = Q(atL, SQ_RHO) * Q(atL, SQ_FS + sp) +
                             0.5 * (S(atL, SL_FS + sp) + qq[sp]);
      sum += specden;
      ql[ES_FS + sp] = specden;
    }
    if (sum < P.small_dens) {
      // The reference falls back to the RIGHT cell's species here
      // (MOL_riemann_K.H:82-86).
#pragma unroll
      for (int sp = 0; sp < NSPEC; ++sp) ql[ES_FS + sp] = Q(at, SQ_FS + sp);
    } else {
      double ys[NSPEC];
      rn_div_group<NSPEC>(ql + ES_FS, sum, ys);
#pragma unroll
      for (int sp = 0; sp < NSPEC; ++sp) ql[ES_FS + sp] = ys[sp];
    }
    ql[ES_RHO] = dmax(sum, P.small_dens);
    ql[ES_REINT] = Q(atL, SQ_REINT) + 0.5 * (S(atL, SL_RE) + qq[NSPEC]);
  }
  {
    const double cspeed = Q(at, SQ_C);
    const double enth = (Q(at, SQ_REINT) + Q(at, SQ_P)) / dmax(Q(at, SQ_RHO), P.small_dens);
    const double d0 = S(at, SL_0), d2 = S(at, SL_2);
    double pr = Q(at, SQ_P) - 0.5 * (d0 + d2) * cspeed;
    qr[ES_P] = dmax(pr, P.small_pres);
    qr[ES_U + d] = Q(at, un) - 0.5 * ((d2 - d0) / Q(at, SQ_RHO));
    qr[ES_U + (t1 - SQ_U)] = Q(at, t1) - 0.5 * S(at, SL_3);
    qr[ES_U + (t2 - SQ_U)] = Q(at, t2) - 0.5 * S(at, SL_4);
    double nq[NSPEC + 1], qq[NSPEC + 1];
#pragma unroll
    for (int sp = 0; sp < NSPEC; ++sp) nq[sp] = Q(at, SQ_FS + sp) * (d0 + d2);
    nq[NSPEC] = enth * (d0 + d2);
    rn_div_group<NSPEC + 1>(nq, cspeed, qq);
    double sum = 0.;
#pragma unroll
    for (int sp = 0; sp < NSPEC; ++sp) {
      const double specden = Q(at, SQ_RHO) * Q(at, SQ_FS + sp) -
                             0.5 * (S(at, SL_FS + sp) + qq[sp]);
      sum += specden;
      qr[ES_FS + sp] = specden;
    }
    if (sum < P.small_dens) {
#pragma unroll
      for (int sp = 0; sp < NSPEC; ++sp) qr[ES_FS + sp] = Q(at, SQ_FS + sp);
    } else {
      double ys[NSPEC];
      rn_div_group<NSPEC>(qr + ES_FS, sum, ys);
#pragma unroll
      for (int sp = 0; sp < NSPEC; ++sp) qr[ES_FS + sp] = ys[sp];
    }
    qr[ES_RHO] = dmax(sum, P.small_dens);
    qr[ES_REINT] = Q(at, SQ_REINT) - 0.5 * (S(at, SL_RE) + qq[NSPEC]);
  }
  const CellAux aL = load_aux(q, s, atL, P.gamma);
  const CellAux aR = load_aux(q, s, at, P.gamma);
  const int idx = (d == 0) ? i : (d == 1) ? j : k;
  cmpflx<d>(ql, qr, aL, aR, idx, g.bclo[d], g.bchi[d], g.dlo[d], g.dhi[d], P, f, qpres, qun);
}

// The MOL edge states of one cell in direction d, from the cell's slopes
// (the halves of mol_riemann_{x,y,z} that read this cell, MOL_riemann_K.H:
// 12-167 and the y/z versions): qr, the state on the cell's low face (the
// right state of that face), complete; and the pieces of the state on its
// high face (the left state of the next face), whose species fall back to
// the next cell's when their sum is below small_dens (the quirk of
// MOL_riemann_K.H:82-86), so the face completes them.
struct MolLeft {
  double p, un, ut1, ut2, reint;
  double spec[NSPEC];
  double sum;
  double c, csml;
};

template <int d>
__device__ __forceinline__ void mol_cell_states(int64_t at, const Space& s, const KParams& P,
                                                const double* q, const double* sl, double* qr,
                                                MolLeft& l) {
  auto Q = [&](int slot) { return ld_ro(q + at + slot * s.sn); };
  constexpr int un = SQ_U + d;
  constexpr int t1 = (d == 0) ? SQ_V : SQ_U;
  constexpr int t2 = (d == 2) ? SQ_V : SQ_W;
  const double cspeed = Q(SQ_C);
  const double enth = (Q(SQ_REINT) + Q(SQ_P)) / dmax(Q(SQ_RHO), P.small_dens);
  const double d0 = sl[SL_0], d2 = sl[SL_2];
  {
    // left state of the next face (this cell as atL)
    const double pl = Q(SQ_P) + 0.5 * (d0 + d2) * cspeed;
    l.p = dmax(pl, P.small_pres);
    l.un = Q(un) + 0.5 * ((d2 - d0) / Q(SQ_RHO));
    l.ut1 = Q(t1) + 0.5 * sl[SL_3];
    l.ut2 = Q(t2) + 0.5 * sl[SL_4];
    double sum = 0.;
#pragma unroll
    for (int sp = 0; sp < NSPEC; ++sp) {
      const double specden =
          Q(SQ_RHO) * Q(SQ_FS + sp) + 0.5 * (sl[SL_FS + sp] + Q(SQ_FS + sp) * (d0 + d2) / cspeed);
      sum += specden;
      l.spec[sp] = specden;
    }
    l.sum = sum;
    l.reint = Q(SQ_REINT) + 0.5 * (sl[SL_RE] + enth * (d0 + d2) / cspeed);
  }
  {
    // right state of this cell's low face (this cell as at)
    const double pr = Q(SQ_P) - 0.5 * (d0 + d2) * cspeed;
    qr[ES_P] = dmax(pr, P.small_pres);
    qr[ES_U + d] = Q(un) - 0.5 * ((d2 - d0) / Q(SQ_RHO));
    qr[ES_U + (t1 - SQ_U)] = Q(t1) - 0.5 * sl[SL_3];
    qr[ES_U + (t2 - SQ_U)] = Q(t2) - 0.5 * sl[SL_4];
    double sum = 0.;
#pragma unroll
    for (int sp = 0; sp < NSPEC; ++sp) {
      const double specden =
          Q(SQ_RHO) * Q(SQ_FS + sp) - 0.5 * (sl[SL_FS + sp] + Q(SQ_FS + sp) * (d0 + d2) / cspeed);
      sum += specden;
      qr[ES_FS + sp] = specden;
    }
    if (sum < P.small_dens) {
#pragma unroll
      for (int sp = 0; sp < NSPEC; ++sp) qr[ES_FS + sp] = Q(SQ_FS + sp);
    } else {
#pragma unroll
      for (int sp = 0; sp < NSPEC; ++sp) qr[ES_FS + sp] = qr[ES_FS + sp] / sum;
    }
    qr[ES_RHO] = dmax(sum, P.small_dens);
    qr[ES_REINT] = Q(SQ_REINT) - 0.5 * (sl[SL_RE] + enth * (d0 + d2) / cspeed);
  }
  l.c = cspeed;
  l.csml = Q(SQ_CSML);
}

// The Riemann flux of the d-face at (i,j,k) from the left pieces of cell
// (i,j,k) - e_d and the right state of cell (i,j,k) (hydro_cmpflx).
template <int d>
__device__ __forceinline__ void mol_face_from_states(int i, int j, int k, const Space& s,
                                                     const KGeom& g, const KParams& P,
                                                     const double* q, const MolLeft& l,
                                                     const double* qr, const CellAux& aR,
                                                     double* f, double& qpres, double& qun) {
  const int64_t at = s.idx(i, j, k);
  constexpr int t1 = (d == 0) ? SQ_V : SQ_U;
  constexpr int t2 = (d == 2) ? SQ_V : SQ_W;
  double ql[ES_N];
  ql[ES_P] = l.p;
  ql[ES_U + d] = l.un;
  ql[ES_U + (t1 - SQ_U)] = l.ut1;
  ql[ES_U + (t2 - SQ_U)] = l.ut2;
  if (l.sum < P.small_dens) {
#pragma unroll
    for (int sp = 0; sp < NSPEC; ++sp) ql[ES_FS + sp] = ld_ro(q + at + (SQ_FS + sp) * s.sn);
  } else {
#pragma unroll
    for (int sp = 0; sp < NSPEC; ++sp) ql[ES_FS + sp] = l.spec[sp] / l.sum;
  }
  ql[ES_RHO] = dmax(l.sum, P.small_dens);
  ql[ES_REINT] = l.reint;
  CellAux aL;
  aL.c = l.c;
  aL.csml = l.csml;
  aL.gamc = P.gamma;
  double qrr[ES_N];
#pragma unroll
  for (int n = 0; n < ES_N; ++n) qrr[n] = qr[n];
  const int idx = (d == 0) ? i : (d == 1) ? j : k;
  cmpflx<d>(ql, qrr, aL, aR, idx, g.bclo[d], g.bchi[d], g.dlo[d], g.dhi[d], P, f, qpres, qun);
}

}  // namespace camr
