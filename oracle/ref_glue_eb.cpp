// Per-box EB hydro of the oracle (test infrastructure): the orchestration of
// hydro_umdrv_eb for do_mol = 1 (Source/Hydro/Hydro_umdrv_eb.cpp:14-191)
// around the reference's own EB kernels, compiled where they lie against the
// AMReX stand-in with AMREX_USE_EB: hydro_ctoprim (Hydro_ctoprim.H:11-101,
// covered cells zeroed as CAMR_construct_hydro_source.cpp:103-111 does),
// MOL_umeth_eb (MOL/MOL_umeth_eb.cpp:21-191), adjust_fluxes_eb
// (Hydro_adjust_fluxes.cpp:48-171), hydro_consup_eb (Hydro_consup.cpp:29-98).
//
// AMReX's ApplyMLRedistribution is not available; its flux redistribution
// ("FluxRedist") is restated here from AMReX's published algorithm
// (apply_flux_redistribution with use_wts_in_divnc = false):
//   for each cut cell c of grow(bx,1):
//     divnc = sum_nb vfrac divc / sum_nb vfrac   (nb: the connected cells of
//             c's 3x3x3 neighbourhood, c included, inside the domain grown
//             by 2 in periodic directions)
//     optmp(c) = (1 - vfrac_c) (divnc - divc_c);  delm(c) = -vfrac_c optmp(c)
//     optmp(nb) += delm(c) wt(nb) / sum_nb (vfrac wt)   for each nb
//   dSdt = divc + optmp on bx (0 on covered cells).
// Neighbour sums run with the z offset outermost and the x offset innermost;
// contributions to one cell arrive in raster order of their sources.
#include <cmath>
#include <cstring>
#include <vector>

#include "Hydro.H"
#include "Hydro_ctoprim.H"
#include "MOL_umeth.H"
#include "Godunov.H"
#include "IndexDefines.H"
#include "oracle_abi.h"

using namespace amrex;

namespace {

Array4<Real> view(double* p, const int lo[3], const int hi[3], int nc) {
  return Array4<Real>(p, IntVect(lo[0], lo[1], lo[2]), IntVect(hi[0] + 1, hi[1] + 1, hi[2] + 1),
                      nc);
}

// ---------------------------------------------------------------------------
// State redistribution (redistribution_type = StateRedist), restated from
// the published method (Berger & Giuliani, "A state redistribution
// algorithm for finite volume schemes on cut cell meshes", J. Comput. Phys.
// 434 (2021) 110205); AMReX's own implementation is not available here, so
// the neighbourhood rule below is this restatement's own:
//   * a cut cell with volume fraction below 1/2 merges with connected,
//     uncovered neighbours of its 3x3x3 block inside the domain (grown in
//     periodic directions), taken in decreasing order of
//     (m . o) / |o| with m = (ap_x(i+1) - ap_x(i), ...) the direction into the
//     fluid and o the neighbour offset (ties in raster order), until the
//     merged volume fraction reaches 1/2 or the neighbourhood holds 8 cells;
//     every other cell's neighbourhood is itself;
//   * N_j: the number of neighbourhoods that hold cell j;
//   * Vhat_i = sum_{j in M_i} vf_j / N_j, xhat_i the matching weighted
//     centroid (cell-width units, x_j = index + cell centroid offset),
//     Qhat_i = sum_{j in M_i} (vf_j / N_j) U*_j / Vhat_i with U* = U + dt divc;
//   * for neighbourhoods of more than one cell, a least-squares gradient of
//     Qhat over the connected neighbours' (xhat, Qhat), limited
//     Barth-Jespersen style so that no member's value leaves the range of
//     those Qhat;
//   * U_new_j = (1/N_j) sum_{i: j in M_i} (Qhat_i + g_i . (x_j - xhat_i)),
//     gathered in raster order of i; dSdt = (U_new - U) / dt (0 on covered
//     cells).
// It conserves sum vf U exactly in exact arithmetic.
constexpr int kSrdMax = 8;

struct SrdNbhd {
  int n;
  int off[kSrdMax];  // offsets as (di+1) + 3(dj+1) + 9(dk+1); off[0] = 13 (the cell)
};

inline void srd_off(int o, int& di, int& dj, int& dk) {
  di = o % 3 - 1;
  dj = (o / 3) % 3 - 1;
  dk = o / 9 - 1;
}

bool srd_inside(const Box& dom, const int* periodic, int i, int j, int k) {
  const int c[3] = {i, j, k};
  for (int d = 0; d < 3; ++d)
    if (!periodic[d] && (c[d] < dom.lo[d] || c[d] > dom.hi[d])) return false;
  return true;
}

SrdNbhd srd_nbhd(const Box& dom, const int* periodic, Array4<EBCellFlag const> const& flag,
                 Array4<const Real> const& vf, const Array4<const Real>* ap, int i, int j,
                 int k) {
  SrdNbhd r;
  r.n = 1;
  r.off[0] = 13;
  const EBCellFlag f = flag(i, j, k);
  if (!f.isSingleValued() || !(vf(i, j, k) < 0.5)) return r;
  const double m0 = ap[0](i + 1, j, k) - ap[0](i, j, k);
  const double m1 = ap[1](i, j + 1, k) - ap[1](i, j, k);
  const double m2 = ap[2](i, j, k + 1) - ap[2](i, j, k);
  int cand[26];
  double score[26];
  int nc = 0;
  for (int kk = -1; kk <= 1; ++kk)
    for (int jj = -1; jj <= 1; ++jj)
      for (int ii = -1; ii <= 1; ++ii) {
        if (ii == 0 && jj == 0 && kk == 0) continue;
        if (!f.isConnected(ii, jj, kk)) continue;
        if (flag(i + ii, j + jj, k + kk).isCovered()) continue;
        if (!srd_inside(dom, periodic, i + ii, j + jj, k + kk)) continue;
        const double len = std::sqrt(double(ii * ii + jj * jj + kk * kk));
        const double sc = (m0 * ii + m1 * jj + m2 * kk) / len;
        // insertion keeps the order: higher score first, raster order on ties
        int at = nc;
        while (at > 0 && score[at - 1] < sc) {
          score[at] = score[at - 1];
          cand[at] = cand[at - 1];
          --at;
        }
        score[at] = sc;
        cand[at] = (ii + 1) + 3 * (jj + 1) + 9 * (kk + 1);
        ++nc;
      }
  double vol = vf(i, j, k);
  for (int c = 0; c < nc && vol < 0.5 && r.n < kSrdMax; ++c) {
    int di, dj, dk;
    srd_off(cand[c], di, dj, dk);
    r.off[r.n++] = cand[c];
    vol += vf(i + di, j + dj, k + dk);
  }
  return r;
}

void state_redistribute(const Box& bx, const Box& dom, const int* periodic,
                        Array4<EBCellFlag const> const& flag, Array4<const Real> const& vf,
                        const Array4<const Real>* ap, Array4<const Real> const& cent,
                        Array4<const Real> const& u, Array4<const Real> const& divc, double dt,
                        Array4<Real> const& out) {
  const Box b4 = amrex::grow(bx, 4), b3 = amrex::grow(bx, 3), b2 = amrex::grow(bx, 2),
            b1 = amrex::grow(bx, 1);
  // neighbourhoods on grow(bx,4)
  const IntVect n4(b4.hi[0] - b4.lo[0] + 1, b4.hi[1] - b4.lo[1] + 1, b4.hi[2] - b4.lo[2] + 1);
  std::vector<SrdNbhd> nb(size_t(n4[0]) * n4[1] * n4[2]);
  auto NB = [&](int i, int j, int k) -> SrdNbhd& {
    return nb[size_t((i - b4.lo[0]) + n4[0] * ((j - b4.lo[1]) + n4[1] * (k - b4.lo[2])))];
  };
  ParallelFor(b4, [&](int i, int j, int k) {
    SrdNbhd& r = NB(i, j, k);
    if (flag(i, j, k).isCovered() || !srd_inside(dom, periodic, i, j, k)) {
      r.n = 0;
      return;
    }
    r = srd_nbhd(dom, periodic, flag, vf, ap, i, j, k);
  });
  auto holds = [&](int i, int j, int k, int di, int dj, int dk) {
    // does the neighbourhood of (i,j,k) hold its neighbour at (di,dj,dk)?
    const SrdNbhd& r = NB(i, j, k);
    const int o = (di + 1) + 3 * (dj + 1) + 9 * (dk + 1);
    for (int c = 0; c < r.n; ++c)
      if (r.off[c] == o) return true;
    return false;
  };
  // N on grow(bx,3)
  FArrayBox Nf(b3, 1), vh(b2, 1), xh(b2, 3), qh(b2, NVAR), gr(b1, 3 * NVAR);
  Nf.setVal(0.0);
  auto N = Nf.array();
  ParallelFor(b3, [&](int i, int j, int k) {
    if (flag(i, j, k).isCovered() || !srd_inside(dom, periodic, i, j, k)) return;
    double cnt = 0.0;
    for (int kk = -1; kk <= 1; ++kk)
      for (int jj = -1; jj <= 1; ++jj)
        for (int ii = -1; ii <= 1; ++ii)
          if (holds(i - ii, j - jj, k - kk, ii, jj, kk)) cnt += 1.0;
    N(i, j, k) = cnt;
  });
  auto VH = vh.array();
  auto XH = xh.array();
  auto QH = qh.array();
  ParallelFor(b2, [&](int i, int j, int k) {
    const SrdNbhd& r = NB(i, j, k);
    if (r.n == 0) return;
    double v = 0.0, x0 = 0.0, x1 = 0.0, x2 = 0.0;
    double q[NVAR];
    for (int n = 0; n < NVAR; ++n) q[n] = 0.0;
    for (int c = 0; c < r.n; ++c) {
      int di, dj, dk;
      srd_off(r.off[c], di, dj, dk);
      const int a = i + di, b = j + dj, cc = k + dk;
      const double w = vf(a, b, cc) / N(a, b, cc);
      v += w;
      x0 += w * (a + cent(a, b, cc, 0));
      x1 += w * (b + cent(a, b, cc, 1));
      x2 += w * (cc + cent(a, b, cc, 2));
      for (int n = 0; n < NVAR; ++n) q[n] += w * (u(a, b, cc, n) + dt * divc(a, b, cc, n));
    }
    VH(i, j, k) = v;
    XH(i, j, k, 0) = x0 / v;
    XH(i, j, k, 1) = x1 / v;
    XH(i, j, k, 2) = x2 / v;
    for (int n = 0; n < NVAR; ++n) QH(i, j, k, n) = q[n] / v;
  });
  auto GR = gr.array();
  ParallelFor(b1, [&](int i, int j, int k) {
    const SrdNbhd& r = NB(i, j, k);
    if (r.n < 2) return;
    const EBCellFlag f = flag(i, j, k);
    double a00 = 0, a01 = 0, a02 = 0, a11 = 0, a12 = 0, a22 = 0;
    for (int kk = -1; kk <= 1; ++kk)
      for (int jj = -1; jj <= 1; ++jj)
        for (int ii = -1; ii <= 1; ++ii) {
          if ((ii == 0 && jj == 0 && kk == 0) || !f.isConnected(ii, jj, kk)) continue;
          if (NB(i + ii, j + jj, k + kk).n == 0) continue;
          const double d0 = XH(i + ii, j + jj, k + kk, 0) - XH(i, j, k, 0);
          const double d1 = XH(i + ii, j + jj, k + kk, 1) - XH(i, j, k, 1);
          const double d2 = XH(i + ii, j + jj, k + kk, 2) - XH(i, j, k, 2);
          a00 += d0 * d0; a01 += d0 * d1; a02 += d0 * d2;
          a11 += d1 * d1; a12 += d1 * d2; a22 += d2 * d2;
        }
    const double c00 = a11 * a22 - a12 * a12, c01 = a02 * a12 - a01 * a22,
                 c02 = a01 * a12 - a02 * a11;
    const double det = a00 * c00 + a01 * c01 + a02 * c02;
    for (int n = 0; n < NVAR; ++n) {
      double g0 = 0.0, g1 = 0.0, g2 = 0.0;
      if (std::fabs(det) > 1e-10) {
        double b0 = 0, b1v = 0, b2v = 0;
        double qmin = QH(i, j, k, n), qmax = QH(i, j, k, n);
        for (int kk = -1; kk <= 1; ++kk)
          for (int jj = -1; jj <= 1; ++jj)
            for (int ii = -1; ii <= 1; ++ii) {
              if ((ii == 0 && jj == 0 && kk == 0) || !f.isConnected(ii, jj, kk)) continue;
              if (NB(i + ii, j + jj, k + kk).n == 0) continue;
              const double d0 = XH(i + ii, j + jj, k + kk, 0) - XH(i, j, k, 0);
              const double d1 = XH(i + ii, j + jj, k + kk, 1) - XH(i, j, k, 1);
              const double d2 = XH(i + ii, j + jj, k + kk, 2) - XH(i, j, k, 2);
              const double dq = QH(i + ii, j + jj, k + kk, n) - QH(i, j, k, n);
              b0 += d0 * dq; b1v += d1 * dq; b2v += d2 * dq;
              qmin = std::min(qmin, QH(i + ii, j + jj, k + kk, n));
              qmax = std::max(qmax, QH(i + ii, j + jj, k + kk, n));
            }
        const double c11 = a00 * a22 - a02 * a02, c12 = a01 * a02 - a00 * a12,
                     c22 = a00 * a11 - a01 * a01;
        g0 = (c00 * b0 + c01 * b1v + c02 * b2v) / det;
        g1 = (c01 * b0 + c11 * b1v + c12 * b2v) / det;
        g2 = (c02 * b0 + c12 * b1v + c22 * b2v) / det;
        double alpha = 1.0;
        for (int c = 0; c < r.n; ++c) {
          int di, dj, dk;
          srd_off(r.off[c], di, dj, dk);
          const int a = i + di, b = j + dj, cc = k + dk;
          const double v = g0 * (a + cent(a, b, cc, 0) - XH(i, j, k, 0)) +
                           g1 * (b + cent(a, b, cc, 1) - XH(i, j, k, 1)) +
                           g2 * (cc + cent(a, b, cc, 2) - XH(i, j, k, 2));
          if (v > 0.0) alpha = std::min(alpha, (qmax - QH(i, j, k, n)) / v);
          else if (v < 0.0) alpha = std::min(alpha, (qmin - QH(i, j, k, n)) / v);
        }
        g0 *= alpha;
        g1 *= alpha;
        g2 *= alpha;
      }
      GR(i, j, k, 3 * n) = g0;
      GR(i, j, k, 3 * n + 1) = g1;
      GR(i, j, k, 3 * n + 2) = g2;
    }
  });
  ParallelFor(bx, [&](int i, int j, int k) {
    if (flag(i, j, k).isCovered()) {
      for (int n = 0; n < NVAR; ++n) out(i, j, k, n) = 0.0;
      return;
    }
    double acc[NVAR];
    for (int n = 0; n < NVAR; ++n) acc[n] = 0.0;
    for (int kk = -1; kk <= 1; ++kk)
      for (int jj = -1; jj <= 1; ++jj)
        for (int ii = -1; ii <= 1; ++ii) {
          const int a = i + ii, b = j + jj, cc = k + kk;
          if (!holds(a, b, cc, -ii, -jj, -kk)) continue;
          if (NB(a, b, cc).n < 2) {
            for (int n = 0; n < NVAR; ++n) acc[n] += QH(a, b, cc, n);
          } else {
            const double x0 = i + cent(i, j, k, 0) - XH(a, b, cc, 0);
            const double x1 = j + cent(i, j, k, 1) - XH(a, b, cc, 1);
            const double x2 = k + cent(i, j, k, 2) - XH(a, b, cc, 2);
            for (int n = 0; n < NVAR; ++n)
              acc[n] += QH(a, b, cc, n) + (GR(a, b, cc, 3 * n) * x0 +
                                           GR(a, b, cc, 3 * n + 1) * x1 +
                                           GR(a, b, cc, 3 * n + 2) * x2);
          }
        }
    for (int n = 0; n < NVAR; ++n) out(i, j, k, n) = (acc[n] / N(i, j, k) - u(i, j, k, n)) / dt;
  });
}

}  // namespace

extern "C" long orc_hydro_box_eb(const orc_params* p, const int bx_lo[3], const int bx_hi[3],
                                 const int dom_lo[3], const int dom_hi[3], const int bclo[3],
                                 const int bchi[3], const int periodic[3], const double* uin,
                                 const int g_lo[3], const int g_hi[3], const unsigned* flag_in,
                                 const double* vfrac_in, const double* ap0, const double* ap1,
                                 const double* ap2, const double* fc0, const double* fc1,
                                 const double* fc2, const double* cent_in, int redist,
                                 int weights_type, double* dsdt, double* flx0, double* flx1,
                                 double* flx2, const double dx_in[3], double dt) {
  shim_assert_count() = 0;
  PassMap pmap;
  init_pass_map(&pmap);
  const PassMap* pm = &pmap;
  const Box bx(IntVect(bx_lo[0], bx_lo[1], bx_lo[2]), IntVect(bx_hi[0], bx_hi[1], bx_hi[2]));
  const Box G(IntVect(g_lo[0], g_lo[1], g_lo[2]), IntVect(g_hi[0], g_hi[1], g_hi[2]));
  const Box dom(IntVect(dom_lo[0], dom_lo[1], dom_lo[2]),
                IntVect(dom_hi[0], dom_hi[1], dom_hi[2]));
  const Geometry geom(dom, periodic);
  auto u = Array4<const Real>(view(const_cast<double*>(uin), g_lo, g_hi, NVAR));
  auto vf = Array4<const Real>(view(const_cast<double*>(vfrac_in), g_lo, g_hi, 1));
  std::vector<EBCellFlag> fl(size_t(G.numPts()));
  for (size_t c = 0; c < fl.size(); ++c) fl[c] = EBCellFlag(flag_in[c]);
  Array4<EBCellFlag const> flag(fl.data(), G.lo, IntVect(g_hi[0] + 1, g_hi[1] + 1, g_hi[2] + 1),
                                1);
  Array4<const Real> ap[3], fc[3];
  const double* aps[3] = {ap0, ap1, ap2};
  const double* fcs[3] = {fc0, fc1, fc2};
  for (int d = 0; d < 3; ++d) {
    int hi[3] = {g_hi[0], g_hi[1], g_hi[2]};
    hi[d] += 1;
    ap[d] = Array4<const Real>(view(const_cast<double*>(aps[d]), g_lo, hi, 1));
    fc[d] = Array4<const Real>(view(const_cast<double*>(fcs[d]), g_lo, hi, 2));
  }
  GpuArray<Real, 3> dx, dxinv;
  for (int d = 0; d < 3; ++d) {
    dx[d] = dx_in[d];
    dxinv[d] = 1. / dx_in[d];
  }
  // q, qaux on grow(bx, numGrow()): 5 for MOL, 6 for Godunov with flux
  // redistribution (CAMR.H:465-472); hydro_ctoprim on the non-covered cells
  const bool mol = p->do_mol != 0;
  // state redistribution needs one more layer of everything
  // (CAMR.H:465-479, CAMR_construct_hydro_source.cpp:146-152)
  const int e_srd = (redist == 2) ? 1 : 0;
  const Box qbx = amrex::grow(bx, (mol ? 5 : 6) + e_srd);
  FArrayBox qf(qbx, QVAR), qauxf(qbx, NQAUX), srcqf(qbx, QVAR), zsrc(qbx, NVAR);
  auto q = qf.array();
  auto qaux = qauxf.array();
  auto srcq = srcqf.array();
  zsrc.setVal(0.0);
  auto src_in = zsrc.const_array();
  ParallelFor(qbx, [=](int i, int j, int k) {
    if (!flag(i, j, k).isCovered()) {
      hydro_ctoprim(i, j, k, u, q, qaux, *pm, p->small_num, p->dual_energy_eta1,
                    p->allow_negative_energy);
    } else {
      for (int n = 0; n < QVAR; n++) q(i, j, k, n) = 0.;
    }
  });
  if (!mol) {
    // sources for the Godunov predictor: zero (no gravity in EB runs here)
    ParallelFor(qbx, [=](int i, int j, int k) {
      if (!flag(i, j, k).isCovered()) {
        hydro_srctoprim(i, j, k, Array4<const Real>(q), Array4<const Real>(qaux), src_in, srcq,
                        *pm);
      } else {
        for (int n = 0; n < QVAR; n++) srcq(i, j, k, n) = 0.;
      }
    });
  }
  const Box bxg_i = amrex::grow(bx, 2 + e_srd);
  const Box bxg_ii = amrex::grow(bxg_i, 1);
  FArrayBox divc(bxg_i, NVAR), redistwgt(bxg_i, 1);
  divc.setVal(0.0);
  redistwgt.setVal(0.0);
  FArrayBox qec[3], flux_tmp[3];
  for (int d = 0; d < 3; ++d) {
    qec[d].resize(amrex::surroundingNodes(amrex::grow(bxg_ii, 1), d), NGDNV);
    flux_tmp[d].resize(amrex::surroundingNodes(bxg_ii, d), NVAR);
    flux_tmp[d].setVal(0.);
  }
  GpuArray<Array4<Real>, 3> qec_arr{{qec[0].array(), qec[1].array(), qec[2].array()}};
  const GpuArray<const Array4<Real>, 3> ft{
      {flux_tmp[0].array(), flux_tmp[1].array(), flux_tmp[2].array()}};
  const int* dl = dom.loVect();
  const int* dh = dom.hiVect();
  auto divc_arr = divc.array();
  auto wt = redistwgt.array();
  if (mol) {
    MOL_umeth_eb(Box(divc_arr), bclo, bchi, dl, dh, Array4<const Real>(q),
                 Array4<const Real>(qaux), qec_arr[0], qec_arr[1], qec_arr[2], flag, dx, ft,
                 p->small, p->small_dens, p->small_pres, p->smallu, p->plm_iorder, pm,
                 weights_type);
  } else {
    Godunov_umeth_eb(Box(divc_arr), bclo, bchi, dl, dh, Array4<const Real>(q),
                     Array4<const Real>(qaux), Array4<const Real>(srcq), ft[0], ft[1], ft[2],
                     qec_arr[0], qec_arr[1], qec_arr[2], ap[0], ap[1], ap[2], flag, dx, dt,
                     p->small, p->small_dens, p->small_pres, p->smallu, p->ppm_type,
                     p->use_pslope, p->use_flattening, p->plm_iorder, pm,
                     p->transverse_reset_density);
  }
  adjust_fluxes_eb(bx, Array4<const Real>(q), u, ap[0], ap[1], ap[2], vf, dx, dxinv, ft, geom,
                   bclo, bchi, p->difmag);
  double* fo[3] = {flx0, flx1, flx2};
  Array4<Real> fout[3];
  for (int d = 0; d < 3; ++d) {
    int hi[3] = {bx_hi[0], bx_hi[1], bx_hi[2]};
    hi[d] += 1;
    fout[d] = view(fo[d], bx_lo, hi, NVAR);
  }
  const GpuArray<const Array4<Real>, 3> fo_arr{{fout[0], fout[1], fout[2]}};
  hydro_consup_eb(bx, Array4<const Real>(q), Array4<const Real>(qaux), divc_arr, wt, qec_arr[0],
                  qec_arr[1], qec_arr[2], ap[0], ap[1], ap[2], fc[0], fc[1], fc[2], vf, flag,
                  dxinv, ft, fo_arr, p->small, p->small_dens, p->small_pres, p->smallu,
                  weights_type);
  auto out = view(dsdt, bx_lo, bx_hi, NVAR);
  if (redist == 2) {
    Array4<const Real> cent;
    std::vector<double> zc;
    if (cent_in) {
      cent = Array4<const Real>(view(const_cast<double*>(cent_in), g_lo, g_hi, 3));
    } else {
      zc.assign(size_t(G.numPts()) * 3, 0.0);
      cent = Array4<const Real>(view(zc.data(), g_lo, g_hi, 3));
    }
    state_redistribute(bx, dom, periodic, flag, vf, ap, cent, u, Array4<const Real>(divc_arr),
                       dt, out);
    return shim_assert_count();
  }
  if (!redist) {
    ParallelFor(bx, NVAR, [=](int i, int j, int k, int n) {
      out(i, j, k, n) = flag(i, j, k).isCovered() ? 0.0 : divc_arr(i, j, k, n);
    });
    return shim_assert_count();
  }
  // flux redistribution
  const Box dbox = geom.growPeriodicDomain(2);
  const Box bxg1 = amrex::grow(bx, 1);
  const Box bxg2 = amrex::grow(bx, 2);
  FArrayBox optf(bxg2, NVAR), delmf(bxg2, NVAR);
  optf.setVal(0.0);
  delmf.setVal(0.0);
  auto optmp = optf.array();
  auto delm = delmf.array();
  ParallelFor(bxg1, NVAR, [=](int i, int j, int k, int n) {
    if (flag(i, j, k).isSingleValued()) {
      Real divnc = 0.0, vtot = 0.0;
      for (int kk = -1; kk <= 1; ++kk)
        for (int jj = -1; jj <= 1; ++jj)
          for (int ii = -1; ii <= 1; ++ii)
            if (flag(i, j, k).isConnected(ii, jj, kk) &&
                dbox.contains(IntVect(i + ii, j + jj, k + kk))) {
              const Real wf = vf(i + ii, j + jj, k + kk);
              vtot += wf;
              divnc += wf * divc_arr(i + ii, j + jj, k + kk, n);
            }
      divnc /= vtot;
      optmp(i, j, k, n) = (1.0 - vf(i, j, k)) * (divnc - divc_arr(i, j, k, n));
      delm(i, j, k, n) = -vf(i, j, k) * optmp(i, j, k, n);
    } else {
      delm(i, j, k, n) = 0.0;
    }
  });
  ParallelFor(bxg1, NVAR, [=](int i, int j, int k, int n) {
    if (flag(i, j, k).isSingleValued()) {
      Real wtot = 0.0;
      for (int kk = -1; kk <= 1; ++kk)
        for (int jj = -1; jj <= 1; ++jj)
          for (int ii = -1; ii <= 1; ++ii)
            if (flag(i, j, k).isConnected(ii, jj, kk) &&
                dbox.contains(IntVect(i + ii, j + jj, k + kk)))
              wtot += vf(i + ii, j + jj, k + kk) * wt(i + ii, j + jj, k + kk);
      wtot = 1.0 / wtot;
      for (int kk = -1; kk <= 1; ++kk)
        for (int jj = -1; jj <= 1; ++jj)
          for (int ii = -1; ii <= 1; ++ii)
            if (flag(i, j, k).isConnected(ii, jj, kk) &&
                dbox.contains(IntVect(i + ii, j + jj, k + kk)))
              optmp(i + ii, j + jj, k + kk, n) += delm(i, j, k, n) * wtot * wt(i + ii, j + jj, k + kk);
    }
  });
  ParallelFor(bx, NVAR, [=](int i, int j, int k, int n) {
    out(i, j, k, n) =
        flag(i, j, k).isCovered() ? 0.0 : divc_arr(i, j, k, n) + optmp(i, j, k, n);
  });
  return shim_assert_count();
}

// ---------------------------------------------------------------------------
// EB level step (MOL or Godunov-PLM), the restated level driver's
// CAMR_advance + post_timestep
// (Source/CAMR_advance.cpp:38-164, Source/CAMR.cpp:679-718) with the EB
// build's guards: covered cells skip enforce_min_density and
// normalize_species (Source/CAMR.cpp:877-891, :960-968), reset_internal_energy
// runs only where rho > 0 (Utils/CAMR_reset_internal_e.H:36-38), computeTemp
// sets T = 0 first (Source/CAMR.cpp:1164-1168), and the CFL minimum skips
// covered cells (:522-540).  The domain is advanced as one box; its ghost
// cells (5, numGrow for MOL + flux redistribution, CAMR.H:455-479) are
// filled as the single-level driver fills them.  Covered cells hold the
// state EB_set_covered gives them at initialisation (zero).
#include "EOS.H"

namespace {

struct LevelEB {
  Box dom, G;
  int periodic[3];
  int bclo[3], bchi[3];
  double dx[3];
  Array4<EBCellFlag const> flag;
};

inline bool covered(const LevelEB& L, int i, int j, int k) { return L.flag(i, j, k).isCovered(); }

// reset_internal_energy on one cell (Utils/CAMR_reset_internal_e.H:13-129),
// skipped where rho <= 0 as the EB build does.
void reset_e_eb(const orc_params* p, Array4<Real> const& S, int i, int j, int k) {
  const Real rho = S(i, j, k, URHO);
  if (!(rho > 0.)) return;
  const Real rhoInv = 1.0 / rho;
  const Real Up = S(i, j, k, UMX) * rhoInv;
  const Real Vp = S(i, j, k, UMY) * rhoInv;
  const Real Wp = S(i, j, k, UMZ) * rhoInv;
  const Real ke = 0.5 * (Up * Up + Vp * Vp + Wp * Wp);
  const Real eden = S(i, j, k, UEDEN) * rhoInv;
  Real massfrac[NUM_SPECIES];
  for (int n = 0; n < NUM_SPECIES; ++n) massfrac[n] = S(i, j, k, n + UFS) * rhoInv;
  Real e_out = 0., small_e = 0.;
  const Real small_T = p->small_temp;
  if (p->allow_small_energy == 0) {
    EOS::RTY2E(rho, small_T, massfrac, small_e);
    if (eden < small_e) {
      if (S(i, j, k, UEINT) * rhoInv < small_e) {
        const Real T = std::max(S(i, j, k, UTEMP), small_T);
        EOS::RTY2E(rho, T, massfrac, e_out);
        S(i, j, k, UEINT) = rho * e_out;
      }
      S(i, j, k, UEDEN) = S(i, j, k, UEINT) + rho * ke;
    } else {
      const Real rho_eint = S(i, j, k, UEDEN) - S(i, j, k, URHO) * ke;
      if (rho_eint > 0. && rho_eint / S(i, j, k, UEDEN) > p->dual_energy_eta2)
        S(i, j, k, UEINT) = rho_eint;
      if (S(i, j, k, UEINT) * rhoInv < small_e) {
        const Real T = std::max(S(i, j, k, UTEMP), small_T);
        EOS::RTY2E(rho, T, massfrac, e_out);
        if (p->dual_energy_update_E_from_e == 1)
          S(i, j, k, UEDEN) += (rho * e_out - S(i, j, k, UEINT));
        S(i, j, k, UEINT) = S(i, j, k, URHO) * e_out;
      }
    }
  } else if (p->allow_negative_energy == 0) {
    if (S(i, j, k, UEDEN) < 0.) {
      if (S(i, j, k, UEINT) < 0.) {
        EOS::RTY2E(rho, small_T, massfrac, e_out);
        S(i, j, k, UEINT) = rho * e_out;
      }
      S(i, j, k, UEDEN) = S(i, j, k, UEINT) + rho * ke;
    } else {
      const Real rho_eint = S(i, j, k, UEDEN) - rho * ke;
      if (rho_eint > 0. && rho_eint / S(i, j, k, UEDEN) > p->dual_energy_eta2) {
        S(i, j, k, UEINT) = rho_eint;
      } else if (S(i, j, k, UEINT) > 0 && p->dual_energy_update_E_from_e == 1) {
        S(i, j, k, UEDEN) = S(i, j, k, UEINT) + rho * ke;
      } else if (S(i, j, k, UEINT) <= 0.) {
        EOS::RTY2E(rho, small_T, massfrac, e_out);
        S(i, j, k, UEINT) = rho * e_out;
        if (p->dual_energy_update_E_from_e == 1)
          S(i, j, k, UEDEN) += (rho * e_out - S(i, j, k, UEINT));
      }
    }
  } else {
    S(i, j, k, UEINT) = S(i, j, k, UEDEN) - rho * ke;
  }
}

void temp_eb(const orc_params* p, Array4<Real> const& S, int i, int j, int k) {
  reset_e_eb(p, S, i, j, k);
  S(i, j, k, UTEMP) = 0.0;
  if (S(i, j, k, URHO) > 0.) {
    const Real rhoInv = 1.0 / S(i, j, k, URHO);
    Real T = S(i, j, k, UTEMP);
    const Real e = S(i, j, k, UEINT) * rhoInv;
    Real massfrac[NUM_SPECIES];
    for (int n = 0; n < NUM_SPECIES; ++n) massfrac[n] = S(i, j, k, UFS + n) * rhoInv;
    const Real rho = S(i, j, k, URHO);
    EOS::REY2T(rho, e, massfrac, T);
    S(i, j, k, UTEMP) = T;
  }
}

void normalize_eb(Array4<Real> const& S, int i, int j, int k) {
  Real sum = 0.;
  for (int n = 0; n < NUM_SPECIES; n++) {
    S(i, j, k, UFS + n) = std::max(std::min(S(i, j, k, URHO), S(i, j, k, UFS + n)), 0.0);
    sum += S(i, j, k, UFS + n);
  }
  if (S(i, j, k, URHO) > 0.) {
    sum /= S(i, j, k, URHO);
    for (int n = 0; n < NUM_SPECIES; n++) S(i, j, k, UFS + n) /= sum;
  }
}

// enforce_min_density over the box `t` (the domain: one tile), skipping
// covered cells; returns the number of cells with zero density.
long enforce_eb(const orc_params* p, const LevelEB& L, Array4<Real> const& S, const Box& t) {
  long nerr = 0;
  ParallelFor(t, [&](int i, int j, int k) {
    if (covered(L, i, j, k)) return;
    if (S(i, j, k, URHO) == 0.) {
      ++nerr;
    } else if (S(i, j, k, URHO) < p->small_dens) {
      Real max_dens = S(i, j, k, URHO);
      int is = i, js = j, ks = k;
      for (int kk = -1; kk <= 1; kk++)
        for (int jj = -1; jj <= 1; jj++)
          for (int ii = -1; ii <= 1; ii++)
            if (t.contains(IntVect(i + ii, j + jj, k + kk)) &&
                S(i + ii, j + jj, k + kk, URHO) > max_dens) {
              is = i + ii; js = j + jj; ks = k + kk;
              max_dens = S(is, js, ks, URHO);
            }
      if (max_dens < p->small_dens) {
        Real massfrac[NUM_SPECIES];
        for (int n = 0; n < NUM_SPECIES; ++n) massfrac[n] = S(i, j, k, UFS + n) / S(i, j, k, URHO);
        Real small_e;
        EOS::RTY2E(p->small_dens, p->small_temp, massfrac, small_e);
        S(i, j, k, URHO) = p->small_dens;
        S(i, j, k, UTEMP) = p->small_temp;
        S(i, j, k, UMX) = 0.;
        S(i, j, k, UMY) = 0.;
        S(i, j, k, UMZ) = 0.;
        S(i, j, k, UEINT) = p->small_dens * small_e;
        S(i, j, k, UEDEN) = S(i, j, k, UEINT);
      } else {
        for (int n = 0; n < NVAR; ++n) S(i, j, k, n) = S(is, js, ks, n);
      }
    }
  });
  return nerr;
}

// The level's boxes are enforce_min_density's windows (its MFIter loop over
// the boxes, Source/CAMR.cpp:960-1043, without tiling as on the GPU).
long enforce_boxes(const orc_params* p, const LevelEB& L, Array4<Real> const& S,
                   const std::vector<Box>& boxes) {
  long nerr = 0;
  for (const Box& b : boxes) nerr += enforce_eb(p, L, S, b);
  return nerr;
}

long clean_eb(const orc_params* p, const LevelEB& L, Array4<Real> const& S,
              const std::vector<Box>& boxes) {
  long nerr = enforce_boxes(p, L, S, boxes);
  ParallelFor(L.dom, [&](int i, int j, int k) {
    if (!covered(L, i, j, k)) normalize_eb(S, i, j, k);
  });
  ParallelFor(L.dom, [&](int i, int j, int k) { temp_eb(p, S, i, j, k); });
  return nerr;
}

// BC kind of component n in direction d for the physical BC word phys
// (Source/Utils/CAMR_setup.cpp:19-21): 1 ext_dir, 2 foextrap, 3 even, 4 odd.
int bc_kind_of(int n, int d, int phys) {
  static const int scalar_bc[] = {0, 1, 2, 3, 3, 3};
  static const int norm_vel_bc[] = {0, 1, 2, 4, 4, 4};
  static const int tang_vel_bc[] = {0, 1, 2, 3, 3, 4};
  if (n == UMX || n == UMY || n == UMZ) return (n - UMX == d) ? norm_vel_bc[phys] : tang_vel_bc[phys];
  return scalar_bc[phys];
}

// expand_state: FillPatch(src) into B over G + clean_state(B).
long expand_eb(const orc_params* p, const LevelEB& L, Array4<Real> const& src,
               Array4<Real> const& B, const std::vector<Box>& boxes) {
  ParallelFor(L.dom, [&](int i, int j, int k) {
    for (int n = 0; n < NVAR; ++n) B(i, j, k, n) = src(i, j, k, n);
  });
  long nerr = enforce_boxes(p, L, B, boxes);
  ParallelFor(L.dom, [&](int i, int j, int k) {
    if (!covered(L, i, j, k)) normalize_eb(B, i, j, k);
  });
  ParallelFor(L.G, [&](int i, int j, int k) {
    const int c[3] = {i, j, k};
    bool inside = true, physical = false;
    int img[3];
    for (int d = 0; d < 3; ++d) {
      img[d] = c[d];
      if (c[d] < L.dom.lo[d] || c[d] > L.dom.hi[d]) {
        inside = false;
        if (L.periodic[d]) {
          const int len = L.dom.hi[d] - L.dom.lo[d] + 1;
          img[d] = L.dom.lo[d] + (((c[d] - L.dom.lo[d]) % len) + len) % len;
        } else {
          physical = true;
        }
      }
    }
    if (inside) return;
    for (int n = 0; n < NVAR; ++n) {
      if (!physical) {
        B(i, j, k, n) = B(img[0], img[1], img[2], n);
        continue;
      }
      int id[3] = {img[0], img[1], img[2]};
      bool neg = false;
      for (int d = 0; d < 3; ++d) {
        if (L.periodic[d]) continue;
        if (id[d] < L.dom.lo[d]) {
          const int t = bc_kind_of(n, d, L.bclo[d]);
          if (t == 1 || t == 2) id[d] = L.dom.lo[d];
          else { id[d] = 2 * L.dom.lo[d] - id[d] - 1; if (t == 4) neg = !neg; }
        } else if (id[d] > L.dom.hi[d]) {
          const int t = bc_kind_of(n, d, L.bchi[d]);
          if (t == 1 || t == 2) id[d] = L.dom.hi[d];
          else { id[d] = 2 * L.dom.hi[d] - id[d] + 1; if (t == 4) neg = !neg; }
        }
      }
      const Real v = src(id[0], id[1], id[2], n);
      B(i, j, k, n) = neg ? -v : v;
    }
  });
  ParallelFor(L.G, [&](int i, int j, int k) { temp_eb(p, B, i, j, k); });
  return nerr;
}

double est_dt_eb(const orc_params* p, const LevelEB& L, Array4<Real> const& S) {
  if (p->fixed_dt > 0.0) return p->fixed_dt;
  double estdt = p->max_dt;
  double estdt_hydro = p->max_dt / p->cfl;
  double dt = std::numeric_limits<double>::max();
  ParallelFor(L.dom, [&](int i, int j, int k) {
    if (covered(L, i, j, k)) return;
    const double rho = S(i, j, k, URHO);
    const double rhoInv = 1.0 / rho;
    const double eint = S(i, j, k, UEINT) / rho;
    const double pres = (p->eos_gamma - 1.0) * rho * eint;
    const double c = std::sqrt(p->eos_gamma * pres / rho);
    dt = std::min(dt, L.dx[0] / (c + std::fabs(S(i, j, k, UMX) * rhoInv)));
    dt = std::min(dt, L.dx[1] / (c + std::fabs(S(i, j, k, UMY) * rhoInv)));
    dt = std::min(dt, L.dx[2] / (c + std::fabs(S(i, j, k, UMZ) * rhoInv)));
  });
  estdt_hydro = std::min(estdt_hydro, dt);
  estdt_hydro *= p->cfl;
  if (estdt_hydro < estdt) estdt = estdt_hydro;
  return estdt;
}

}  // namespace

// One all-regular box of an EB level: construct_hydro_source's regular
// branch in an EB build (CAMR_construct_hydro_source.cpp:81-120, :225-238):
// q on grow(bx, numGrow() = 5) with covered cells zero, then the
// reference's regular hydro_umdrv accumulating into dsdt.
static long eb_regular_box(const orc_params* p, const LevelEB& L, const Box& bx,
                    Array4<Real> const& B, Array4<Real> const& dsdt, double dt) {
  const Box qbx = amrex::grow(bx, p->do_mol ? 5 : 6);
  PassMap pmap;
  init_pass_map(&pmap);
  FArrayBox q(qbx, QVAR), qaux(qbx, NQAUX), src_q(qbx, QVAR);
  auto qarr = q.array();
  auto qauxar = qaux.array();
  auto srcqarr = src_q.array();
  Array4<const Real> sarr(B);
  const Real small_num = p->small_num;
  const Real eta1 = p->dual_energy_eta1;
  const int ane = p->allow_negative_energy;
  ParallelFor(qbx, [&](int i, int j, int k) {
    if (!covered(L, i, j, k)) {
      hydro_ctoprim(i, j, k, sarr, qarr, qauxar, pmap, small_num, eta1, ane);
    } else {
      for (int n = 0; n < QVAR; ++n) qarr(i, j, k, n) = 0.;
    }
  });
  if (!p->do_mol) {
    FArrayBox zsrc(qbx, NVAR);
    zsrc.setVal(0.0);
    auto src_in = zsrc.const_array();
    ParallelFor(qbx, [&](int i, int j, int k) {
      if (!covered(L, i, j, k)) {
        hydro_srctoprim(i, j, k, Array4<const Real>(qarr), Array4<const Real>(qauxar), src_in,
                        srcqarr, pmap);
      } else {
        for (int n = 0; n < QVAR; ++n) srcqarr(i, j, k, n) = 0.;
      }
    });
  }
  FArrayBox flux[3], area[3], vol(bx, 1);
  Array4<Real> fa[3];
  Array4<Real> aa[3];
  for (int d = 0; d < 3; ++d) {
    const Box efbx = amrex::surroundingNodes(bx, d);
    flux[d].resize(efbx, NVAR);
    flux[d].setVal(0.0);
    fa[d] = flux[d].array();
    area[d].resize(efbx, 1);
    area[d].setVal((d == 0) ? L.dx[1] * L.dx[2] : (d == 1) ? L.dx[0] * L.dx[2] : L.dx[0] * L.dx[1]);
    aa[d] = area[d].array();
  }
  vol.setVal(L.dx[0] * L.dx[1] * L.dx[2]);
  const amrex::GpuArray<const Array4<Real>, 3> flx_arr{{fa[0], fa[1], fa[2]}};
  const amrex::GpuArray<const Array4<const Real>, 3> a{
      {Array4<const Real>(aa[0]), Array4<const Real>(aa[1]), Array4<const Real>(aa[2])}};
  const amrex::GpuArray<Real, 3> dxa{{L.dx[0], L.dx[1], L.dx[2]}};
  const Geometry geom(L.dom, L.periodic);
  hydro_umdrv(p->do_mol != 0, bx, geom, L.bclo, L.bchi, sarr, dsdt, qarr, qauxar, srcqarr, dxa, dt,
              p->ppm_type, p->plm_iorder, p->use_pslope, p->use_flattening,
              p->transverse_reset_density, p->small, p->small_dens, p->small_pres, p->smallu,
              p->difmag, flx_arr, a, vol.array(), &pmap);
  return 0;
}

extern "C" long orc_eb_advance(const orc_params* p, const orc_level* lev, const unsigned* flag_in,
                               const double* vfrac, const double* ap0, const double* ap1,
                               const double* ap2, const double* fc0, const double* fc1,
                               const double* fc2, const double* cent, double* state, int nsteps,
                               int first_step, double* dt_prev, double* dt_hist, int redist) {
  LevelEB L;
  for (int d = 0; d < 3; ++d) {
    L.dom.lo[d] = lev->dom_lo[d];
    L.dom.hi[d] = lev->dom_hi[d];
    L.periodic[d] = lev->is_periodic[d];
    L.bclo[d] = lev->bc_lo[d];
    L.bchi[d] = lev->bc_hi[d];
    L.dx[d] = lev->dx[d];
  }
  // ghost cells: numGrow() with flux redistribution, 5 for MOL, 6 for
  // Godunov (CAMR.H:465-472); the geometry covers grow(domain, ng)
  const int ng = (p->do_mol ? 5 : 6) + (redist == 2 ? 1 : 0);
  L.G = amrex::grow(L.dom, ng);
  std::vector<EBCellFlag> fl(size_t(L.G.numPts()));
  for (size_t c = 0; c < fl.size(); ++c) fl[c] = EBCellFlag(flag_in[c]);
  L.flag = Array4<EBCellFlag const>(fl.data(), L.G.lo,
                                    IntVect(L.G.hi[0] + 1, L.G.hi[1] + 1, L.G.hi[2] + 1), 1);
  auto S = view(state, L.dom.lo.v, L.dom.hi.v, NVAR);
  FArrayBox Sold_f(L.dom, NVAR), B_f(L.G, NVAR), B2_f(L.G, NVAR), d1_f(L.dom, NVAR),
      d2_f(L.dom, NVAR);
  auto S_old = Sold_f.array();
  auto B = B_f.array();
  auto B2 = B2_f.array();
  auto k1 = d1_f.array();
  auto k2 = d2_f.array();
  const int g_lo[3] = {L.G.lo[0], L.G.lo[1], L.G.lo[2]};
  const int g_hi[3] = {L.G.hi[0], L.G.hi[1], L.G.hi[2]};
  const int* dlo = L.dom.lo.v;
  const int* dhi = L.dom.hi.v;
  // the level's boxes (max_grid_size chop from the low end) and their kind
  // (CAMR_construct_hydro_source.cpp:76-78, :150-153): 0 covered (skipped),
  // 1 grow(bx,2) all regular (regular hydro), 2 cut (hydro_umdrv_eb)
  std::vector<Box> boxes;
  std::vector<int> kind;
  {
    int step[3];
    for (int d = 0; d < 3; ++d) {
      const int n = L.dom.hi[d] - L.dom.lo[d] + 1;
      step[d] = lev->max_grid_size[d] > 0 ? lev->max_grid_size[d] : n;
    }
    for (int k = L.dom.lo[2]; k <= L.dom.hi[2]; k += step[2])
      for (int j = L.dom.lo[1]; j <= L.dom.hi[1]; j += step[1])
        for (int i = L.dom.lo[0]; i <= L.dom.hi[0]; i += step[0]) {
          const Box b(IntVect(i, j, k),
                      IntVect(std::min(i + step[0] - 1, L.dom.hi[0]),
                              std::min(j + step[1] - 1, L.dom.hi[1]),
                              std::min(k + step[2] - 1, L.dom.hi[2])));
          bool all_cov = true, all_reg = true;
          ParallelFor(b, [&](int ii, int jj, int kk) {
            if (!covered(L, ii, jj, kk)) all_cov = false;
          });
          ParallelFor(amrex::grow(b, redist == 2 ? 3 : 2), [&](int ii, int jj, int kk) {
            if (!L.flag(ii, jj, kk).isRegular()) all_reg = false;
          });
          boxes.push_back(b);
          kind.push_back(all_cov ? 0 : (all_reg ? 1 : 2));
        }
  }
  // construct_hydro_source of one stage: src_to_fill = 0, then each box
  auto stage = [&](Array4<Real> const& Bv, Array4<Real> const& kout, double dt) -> long {
    long ne = 0;
    ParallelFor(L.dom, NVAR, [&](int i, int j, int k, int n) { kout(i, j, k, n) = 0.0; });
    for (size_t b = 0; b < boxes.size(); ++b) {
      const Box& bx = boxes[b];
      if (kind[b] == 0) continue;
      if (kind[b] == 1) {
        ne += eb_regular_box(p, L, bx, Bv, kout, dt);
        continue;
      }
      FArrayBox dfab(bx, NVAR), ff[3];
      for (int d = 0; d < 3; ++d) ff[d].resize(amrex::surroundingNodes(bx, d), NVAR);
      ne += orc_hydro_box_eb(p, bx.lo.v, bx.hi.v, dlo, dhi, L.bclo, L.bchi, L.periodic, Bv.p,
                             g_lo, g_hi, flag_in, vfrac, ap0, ap1, ap2, fc0, fc1, fc2, cent,
                             redist,
                             p->eb_weights_type, dfab.array().p, ff[0].array().p,
                             ff[1].array().p, ff[2].array().p, L.dx, dt);
      auto dv = dfab.array();
      ParallelFor(bx, NVAR, [&](int i, int j, int k, int n) { kout(i, j, k, n) = dv(i, j, k, n); });
    }
    return ne;
  };
  long nerr = 0;
  double dt_level = *dt_prev;
  for (int step = 0; step < nsteps; ++step) {
    double dt;
    const double est = est_dt_eb(p, L, S);
    if (first_step && step == 0) {
      const double init_dt = (p->initial_dt > 0.0) ? p->initial_dt : p->init_shrink * est;
      dt = std::min(std::numeric_limits<double>::max(), 1 * init_dt) / 1;
    } else {
      double dt_min = est;
      if (p->fixed_dt <= 0.0) dt_min = std::min(dt_min, p->change_max * dt_level);
      dt = std::min(std::numeric_limits<double>::max(), 1 * dt_min) / 1;
    }
    ParallelFor(L.dom, NVAR, [&](int i, int j, int k, int n) { S_old(i, j, k, n) = S(i, j, k, n); });
    nerr += clean_eb(p, L, S_old, boxes);
    nerr += expand_eb(p, L, S_old, B, boxes);
    ParallelFor(L.dom, NVAR, [&](int i, int j, int k, int n) { S(i, j, k, n) = B(i, j, k, n); });
    if (p->add_grav_src) {
      ParallelFor(L.dom, [&](int i, int j, int k) {
        Real src[NVAR];
        for (int n = 0; n < NVAR; ++n) src[n] = 0.0;
        src[UMZ] = p->const_grav * S_old(i, j, k, URHO);
        src[UEDEN] = p->const_grav * S_old(i, j, k, UMZ);
        for (int n = 0; n < NVAR; ++n) S(i, j, k, n) += dt * src[n];
      });
    }
    nerr += stage(B, k1, dt);
    ParallelFor(L.dom, NVAR, [&](int i, int j, int k, int n) { S(i, j, k, n) += dt * k1(i, j, k, n); });
    if (p->do_mol) {
      nerr += expand_eb(p, L, S, B2, boxes);
      nerr += stage(B2, k2, dt);
      ParallelFor(L.dom, NVAR, [&](int i, int j, int k, int n) {
        S(i, j, k, n) = 0.5 * B2(i, j, k, n) + 0.5 * S_old(i, j, k, n);
      });
      ParallelFor(L.dom, NVAR, [&](int i, int j, int k, int n) {
        S(i, j, k, n) += 0.5 * dt * k2(i, j, k, n);
      });
    }
    nerr += clean_eb(p, L, S, boxes);
    if (p->add_grav_src) {
      ParallelFor(L.dom, [&](int i, int j, int k) {
        Real src[NVAR];
        for (int n = 0; n < NVAR; ++n) src[n] = 0.0;
        src[UMZ] = 0.5 * p->const_grav * (S(i, j, k, URHO) - S_old(i, j, k, URHO));
        src[UEDEN] = 0.5 * p->const_grav * (S(i, j, k, UMZ) - S_old(i, j, k, UMZ));
        for (int n = 0; n < NVAR; ++n) S(i, j, k, n) += dt * src[n];
      });
      nerr += clean_eb(p, L, S, boxes);
    }
    nerr += clean_eb(p, L, S, boxes);
    dt_level = dt;
    if (dt_hist) dt_hist[step] = dt;
  }
  *dt_prev = dt_level;
  return nerr;
}

// initData's epilogue in the EB build (Source/CAMR.cpp:414-420):
// enforce_consistent_e where rho > 0 (:910-939), then computeTemp.
extern "C" void orc_eb_init_finalize(const orc_params* p, const orc_level* lev, double* state) {
  const int* lo = lev->dom_lo;
  const int* hi = lev->dom_hi;
  auto S = view(state, lo, hi, NVAR);
  const Box dom(IntVect(lo[0], lo[1], lo[2]), IntVect(hi[0], hi[1], hi[2]));
  ParallelFor(dom, [&](int i, int j, int k) {
    if (S(i, j, k, URHO) > 0.) {
      const Real rhoInv = 1.0 / S(i, j, k, URHO);
      const Real u = S(i, j, k, UMX) * rhoInv;
      const Real v = S(i, j, k, UMY) * rhoInv;
      const Real w = S(i, j, k, UMZ) * rhoInv;
      S(i, j, k, UEDEN) = S(i, j, k, UEINT) + 0.5 * S(i, j, k, URHO) * (u * u + v * v + w * w);
    }
  });
  ParallelFor(dom, [&](int i, int j, int k) { temp_eb(p, S, i, j, k); });
}
