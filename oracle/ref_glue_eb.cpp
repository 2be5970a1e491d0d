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
#include "IndexDefines.H"
#include "oracle_abi.h"

using namespace amrex;

namespace {

Array4<Real> view(double* p, const int lo[3], const int hi[3], int nc) {
  return Array4<Real>(p, IntVect(lo[0], lo[1], lo[2]), IntVect(hi[0] + 1, hi[1] + 1, hi[2] + 1),
                      nc);
}

}  // namespace

extern "C" long orc_hydro_box_eb(const orc_params* p, const int bx_lo[3], const int bx_hi[3],
                                 const int dom_lo[3], const int dom_hi[3], const int bclo[3],
                                 const int bchi[3], const int periodic[3], const double* uin,
                                 const int g_lo[3], const int g_hi[3], const unsigned* flag_in,
                                 const double* vfrac_in, const double* ap0, const double* ap1,
                                 const double* ap2, const double* fc0, const double* fc1,
                                 const double* fc2, int redist, int weights_type, double* dsdt,
                                 double* flx0, double* flx1, double* flx2, const double dx_in[3],
                                 double dt) {
  (void)dt;
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
  // q, qaux on grow(bx, 5): hydro_ctoprim on the non-covered cells
  const Box qbx = amrex::grow(bx, 5);
  FArrayBox qf(qbx, QVAR), qauxf(qbx, NQAUX);
  auto q = qf.array();
  auto qaux = qauxf.array();
  ParallelFor(qbx, [=](int i, int j, int k) {
    if (!flag(i, j, k).isCovered()) {
      hydro_ctoprim(i, j, k, u, q, qaux, *pm, p->small_num, p->dual_energy_eta1,
                    p->allow_negative_energy);
    } else {
      for (int n = 0; n < QVAR; n++) q(i, j, k, n) = 0.;
    }
  });
  const Box bxg_i = amrex::grow(bx, 2);
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
  MOL_umeth_eb(Box(divc_arr), bclo, bchi, dl, dh, Array4<const Real>(q), Array4<const Real>(qaux),
               qec_arr[0], qec_arr[1], qec_arr[2], flag, dx, ft, p->small, p->small_dens,
               p->small_pres, p->smallu, p->plm_iorder, pm, weights_type);
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
