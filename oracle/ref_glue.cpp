// C entry points around the reference's own per-box hydro code, compiled on
// the CPU against the repo's AMReX stand-in (oracle/amrex_shim).  This file is
// test infrastructure: it is linked only into oracle/_ref/libcamr_ref.so,
// which tests and the CPU-baseline leg of bench.py load to pin the oracle
// restatement and the CUDA kernels against the reference itself.
//
// What one call does mirrors one MFIter iteration of
// CAMR::construct_hydro_source (Source/Hydro/CAMR_construct_hydro_source.cpp:71-254):
//   flux[d].setVal(0) on surroundingNodes(bx,d)            (:84-89)
//   q, qaux, src_q on grow(bx, 4)                          (:95-97)
//   hydro_ctoprim over grow(bx, 4)                         (:108-120)
//   hydro_srctoprim over grow(bx, 4) when !do_mol          (:129-143)
//   hydro_umdrv(...)                                       (:233-238)
// dsdt is accumulated (+=) exactly as the reference does.
#include <cstdint>
#include <cstring>

#include "oracle_abi.h"

#include "Hydro.H"
#include "Hydro_ctoprim.H"
#include "IndexDefines.H"

using amrex::Array4;
using amrex::Box;
using amrex::IntVect;
using amrex::Real;

namespace {

Array4<Real> make_arr(double* p, const int* lo, const int* hi, int nc) {
  return Array4<Real>(p, IntVect(lo[0], lo[1], lo[2]),
                      IntVect(hi[0] + 1, hi[1] + 1, hi[2] + 1), nc);
}

}  // namespace

extern "C" {

// The oracle ABI's per-box hydro, implemented with the reference's own
// hydro_ctoprim / hydro_srctoprim / hydro_umdrv.
long orc_hydro_box(const orc_params* p, const int bx_lo[3], const int bx_hi[3],
                   const int dom_lo[3], const int dom_hi[3], const int bclo[3],
                   const int bchi[3], const double* uin, const int uin_lo[3],
                   const int uin_hi[3], const double* src, double* dsdt,
                   const int dsdt_lo[3], const int dsdt_hi[3], double* flx0,
                   double* flx1, double* flx2, const double dx[3], double dt) {
  amrex::shim_assert_count() = 0;
  const Box bx(IntVect(bx_lo[0], bx_lo[1], bx_lo[2]),
               IntVect(bx_hi[0], bx_hi[1], bx_hi[2]));
  const Box qbx = amrex::grow(bx, 4);
  amrex::Geometry geom(Box(IntVect(dom_lo[0], dom_lo[1], dom_lo[2]),
                           IntVect(dom_hi[0], dom_hi[1], dom_hi[2])));

  auto uarr = make_arr(const_cast<double*>(uin), uin_lo, uin_hi, NVAR);
  Array4<const Real> sarr(uarr);
  auto hyd_src = make_arr(dsdt, dsdt_lo, dsdt_hi, NVAR);

  double* fp[3] = {flx0, flx1, flx2};
  amrex::FArrayBox area_fab[3], vol_fab;
  Array4<Real> flxa[3];
  Array4<Real> areaa[3];
  for (int d = 0; d < 3; ++d) {
    const Box efbx = amrex::surroundingNodes(bx, d);
    flxa[d] = make_arr(fp[d], efbx.lo.v, efbx.hi.v, NVAR);
    auto fa = flxa[d];
    amrex::ParallelFor(efbx, [=](int i, int j, int k) {
      for (int n = 0; n < NVAR; ++n) fa(i, j, k, n) = 0.0;
    });
    area_fab[d].resize(efbx, 1);
    // Cartesian face area as AMReX's CoordSys computes it.
    const double a = (d == 0) ? dx[1] * dx[2] : (d == 1) ? dx[0] * dx[2] : dx[0] * dx[1];
    area_fab[d].setVal(a);
    areaa[d] = area_fab[d].array();
  }
  vol_fab.resize(bx, 1);
  vol_fab.setVal(dx[0] * dx[1] * dx[2]);
  Array4<Real> vola = vol_fab.array();

  amrex::FArrayBox q(qbx, QVAR), qaux(qbx, NQAUX), src_q(qbx, QVAR);
  auto qarr = q.array();
  auto qauxar = qaux.array();
  auto srcqarr = src_q.array();

  PassMap pmap;
  init_pass_map(&pmap);

  const Real small_num = p->small_num;
  const Real eta1 = p->dual_energy_eta1;
  const int ane = p->allow_negative_energy;
  amrex::ParallelFor(qbx, [=](int i, int j, int k) {
    hydro_ctoprim(i, j, k, sarr, qarr, qauxar, pmap, small_num, eta1, ane);
  });

  amrex::FArrayBox zero_src;
  Array4<const Real> src_in;
  if (src) {
    src_in = Array4<const Real>(make_arr(const_cast<double*>(src), uin_lo, uin_hi, NVAR));
  } else {
    zero_src.resize(qbx, NVAR);
    zero_src.setVal(0.0);
    src_in = zero_src.const_array();
  }
  if (!p->do_mol) {
    amrex::ParallelFor(qbx, [=](int i, int j, int k) {
      hydro_srctoprim(i, j, k, qarr, qauxar, src_in, srcqarr, pmap);
    });
  }

  const amrex::GpuArray<const Array4<Real>, 3> flx_arr{{flxa[0], flxa[1], flxa[2]}};
  const amrex::GpuArray<const Array4<const Real>, 3> a{
      {Array4<const Real>(areaa[0]), Array4<const Real>(areaa[1]),
       Array4<const Real>(areaa[2])}};
  const amrex::GpuArray<Real, 3> dxa{{dx[0], dx[1], dx[2]}};

  hydro_umdrv(p->do_mol != 0, bx, geom, bclo, bchi, sarr, hyd_src, qarr,
              qauxar, srcqarr, dxa, dt, p->ppm_type, p->plm_iorder,
              p->use_pslope, p->use_flattening, p->transverse_reset_density,
              p->small, p->small_dens, p->small_pres, p->smallu, p->difmag,
              flx_arr, a, vola, &pmap);
  return amrex::shim_assert_count();
}

// The reference's hydro_ctoprim (and, for CTU, hydro_srctoprim of `src`,
// NULL = zero) over the region [lo, hi] of uin: q (QVAR), qaux (NQAUX) and
// src_q (QVAR) on that region, as construct_hydro_source computes them
// (Source/Hydro/CAMR_construct_hydro_source.cpp:108-143).
long orc_ref_ctoprim(const orc_params* p, const int lo[3], const int hi[3], const double* uin,
                     const int uin_lo[3], const int uin_hi[3], const double* src, double* q,
                     double* qaux, double* srcq) {
  amrex::shim_assert_count() = 0;
  const Box qbx(IntVect(lo[0], lo[1], lo[2]), IntVect(hi[0], hi[1], hi[2]));
  Array4<const Real> sarr(make_arr(const_cast<double*>(uin), uin_lo, uin_hi, NVAR));
  auto qarr = make_arr(q, lo, hi, QVAR);
  auto qauxar = make_arr(qaux, lo, hi, NQAUX);
  auto srcqarr = make_arr(srcq, lo, hi, QVAR);
  PassMap pmap;
  init_pass_map(&pmap);
  const Real small_num = p->small_num;
  const Real eta1 = p->dual_energy_eta1;
  const int ane = p->allow_negative_energy;
  amrex::ParallelFor(qbx, [=](int i, int j, int k) {
    hydro_ctoprim(i, j, k, sarr, qarr, qauxar, pmap, small_num, eta1, ane);
  });
  amrex::FArrayBox zero_src;
  Array4<const Real> src_in;
  if (src) {
    src_in = Array4<const Real>(make_arr(const_cast<double*>(src), uin_lo, uin_hi, NVAR));
  } else {
    zero_src.resize(qbx, NVAR);
    zero_src.setVal(0.0);
    src_in = zero_src.const_array();
  }
  amrex::ParallelFor(qbx, [=](int i, int j, int k) {
    hydro_srctoprim(i, j, k, qarr, qauxar, src_in, srcqarr, pmap);
  });
  return amrex::shim_assert_count();
}

// The reference's hydro_umdrv with every input given by the caller: q and
// qaux on grow(bx,4) (layout of orc_ref_ctoprim), src_q (NULL = zero),
// face areas area[d] on surroundingNodes(bx,d) and volumes on bx (NULL =
// Cartesian from dx).  flx[d] are zeroed first; dsdt is accumulated.
long orc_ref_hydro_box_full(const orc_params* p, const int bx_lo[3], const int bx_hi[3],
                            const int dom_lo[3], const int dom_hi[3], const int bclo[3],
                            const int bchi[3], const double* uin, const int uin_lo[3],
                            const int uin_hi[3], const double* q, const double* qaux,
                            const double* srcq, const double* area0, const double* area1,
                            const double* area2, const double* vol, double* dsdt,
                            double* flx0, double* flx1, double* flx2, const double dx[3],
                            double dt) {
  amrex::shim_assert_count() = 0;
  const Box bx(IntVect(bx_lo[0], bx_lo[1], bx_lo[2]), IntVect(bx_hi[0], bx_hi[1], bx_hi[2]));
  const Box qbx = amrex::grow(bx, 4);
  amrex::Geometry geom(Box(IntVect(dom_lo[0], dom_lo[1], dom_lo[2]),
                           IntVect(dom_hi[0], dom_hi[1], dom_hi[2])));
  Array4<const Real> sarr(make_arr(const_cast<double*>(uin), uin_lo, uin_hi, NVAR));
  auto hyd_src = make_arr(dsdt, bx.lo.v, bx.hi.v, NVAR);
  double* fp[3] = {flx0, flx1, flx2};
  const double* ap[3] = {area0, area1, area2};
  amrex::FArrayBox area_fab[3], vol_fab, zero_srcq;
  Array4<Real> flxa[3];
  Array4<Real> areaa[3];
  for (int d = 0; d < 3; ++d) {
    const Box efbx = amrex::surroundingNodes(bx, d);
    flxa[d] = make_arr(fp[d], efbx.lo.v, efbx.hi.v, NVAR);
    auto fa = flxa[d];
    amrex::ParallelFor(efbx, [=](int i, int j, int k) {
      for (int n = 0; n < NVAR; ++n) fa(i, j, k, n) = 0.0;
    });
    if (ap[d]) {
      areaa[d] = make_arr(const_cast<double*>(ap[d]), efbx.lo.v, efbx.hi.v, 1);
    } else {
      area_fab[d].resize(efbx, 1);
      const double a = (d == 0) ? dx[1] * dx[2] : (d == 1) ? dx[0] * dx[2] : dx[0] * dx[1];
      area_fab[d].setVal(a);
      areaa[d] = area_fab[d].array();
    }
  }
  Array4<Real> vola;
  if (vol) {
    vola = make_arr(const_cast<double*>(vol), bx.lo.v, bx.hi.v, 1);
  } else {
    vol_fab.resize(bx, 1);
    vol_fab.setVal(dx[0] * dx[1] * dx[2]);
    vola = vol_fab.array();
  }
  Array4<const Real> qarr(make_arr(const_cast<double*>(q), qbx.lo.v, qbx.hi.v, QVAR));
  Array4<const Real> qauxar(make_arr(const_cast<double*>(qaux), qbx.lo.v, qbx.hi.v, NQAUX));
  Array4<const Real> srcqarr;
  if (srcq) {
    srcqarr = Array4<const Real>(make_arr(const_cast<double*>(srcq), qbx.lo.v, qbx.hi.v, QVAR));
  } else {
    zero_srcq.resize(qbx, QVAR);
    zero_srcq.setVal(0.0);
    srcqarr = zero_srcq.const_array();
  }
  PassMap pmap;
  init_pass_map(&pmap);
  const amrex::GpuArray<const Array4<Real>, 3> flx_arr{{flxa[0], flxa[1], flxa[2]}};
  const amrex::GpuArray<const Array4<const Real>, 3> a{
      {Array4<const Real>(areaa[0]), Array4<const Real>(areaa[1]),
       Array4<const Real>(areaa[2])}};
  const amrex::GpuArray<Real, 3> dxa{{dx[0], dx[1], dx[2]}};
  hydro_umdrv(p->do_mol != 0, bx, geom, bclo, bchi, sarr, hyd_src, qarr, qauxar, srcqarr, dxa,
              dt, p->ppm_type, p->plm_iorder, p->use_pslope, p->use_flattening,
              p->transverse_reset_density, p->small, p->small_dens, p->small_pres, p->smallu,
              p->difmag, flx_arr, a, vola, &pmap);
  return amrex::shim_assert_count();
}

}  // extern "C"
