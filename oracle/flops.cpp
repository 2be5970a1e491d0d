// Algorithmic flop count of the reference's per-box hydro: its own
// hydro_ctoprim, hydro_srctoprim and hydro_umdrv (compiled unmodified with
// amrex::Real = a counting double, CAMR_FLOP_COUNT) run on one box, the
// operations counted.  Test and measurement infrastructure: linked only into
// oracle/_ref/libcamr_ref_flops.so, which bench.py's measurement legs and a
// CPU test load.
//
// One call mirrors one MFIter iteration of CAMR::construct_hydro_source
// (Source/Hydro/CAMR_construct_hydro_source.cpp:71-254) on the box [0, n-1]
// with zero sources and Cartesian metrics; counts[6] receives adds (incl.
// subtractions), multiplies, divisions, square roots, comparisons and
// abs/copysign.
#include <cstring>

#include "oracle_abi.h"

#include "Hydro.H"
#include "Hydro_ctoprim.H"
#include "IndexDefines.H"

using amrex::Array4;
using amrex::Box;
using amrex::IntVect;
using amrex::Real;

extern "C" long orc_count_flops(const orc_params* p, const int n[3], const int bclo[3],
                                const int bchi[3], const double* uin, const double dx[3],
                                double dt, long long counts[6]) {
  amrex::shim_assert_count() = 0;
  const Box bx(IntVect(0, 0, 0), IntVect(n[0] - 1, n[1] - 1, n[2] - 1));
  const Box qbx = amrex::grow(bx, 4);
  amrex::Geometry geom(bx);
  // uin: NVAR comps on grow(bx, 4), i fastest, copied into counting fabs
  amrex::FArrayBox ufab(qbx, NVAR);
  auto u = ufab.array();
  {
    long m = 0;
    for (int c = 0; c < NVAR; ++c)
      for (int k = qbx.lo[2]; k <= qbx.hi[2]; ++k)
        for (int j = qbx.lo[1]; j <= qbx.hi[1]; ++j)
          for (int i = qbx.lo[0]; i <= qbx.hi[0]; ++i) u(i, j, k, c) = Real(uin[m++]);
  }
  Array4<const Real> sarr(u);
  amrex::FArrayBox dsdt(bx, NVAR), flux[3], area[3], vol(bx, 1);
  dsdt.setVal(0.0);
  Array4<Real> fa[3], aa[3];
  for (int d = 0; d < 3; ++d) {
    const Box efbx = amrex::surroundingNodes(bx, d);
    flux[d].resize(efbx, NVAR);
    flux[d].setVal(0.0);
    fa[d] = flux[d].array();
    area[d].resize(efbx, 1);
    area[d].setVal((d == 0) ? dx[1] * dx[2] : (d == 1) ? dx[0] * dx[2] : dx[0] * dx[1]);
    aa[d] = area[d].array();
  }
  vol.setVal(dx[0] * dx[1] * dx[2]);
  amrex::FArrayBox q(qbx, QVAR), qaux(qbx, NQAUX), src_q(qbx, QVAR), zero_src(qbx, NVAR);
  zero_src.setVal(0.0);
  auto qarr = q.array();
  auto qauxar = qaux.array();
  auto srcqarr = src_q.array();
  auto src_in = zero_src.const_array();
  PassMap pmap;
  init_pass_map(&pmap);
  const Real small_num = p->small_num;
  const Real eta1 = p->dual_energy_eta1;
  const int ane = p->allow_negative_energy;
  camr_flops::counts() = camr_flops::Counts{};
  amrex::ParallelFor(qbx, [=](int i, int j, int k) {
    hydro_ctoprim(i, j, k, sarr, qarr, qauxar, pmap, small_num, eta1, ane);
  });
  if (!p->do_mol) {
    amrex::ParallelFor(qbx, [=](int i, int j, int k) {
      hydro_srctoprim(i, j, k, qarr, qauxar, src_in, srcqarr, pmap);
    });
  }
  const amrex::GpuArray<const Array4<Real>, 3> flx_arr{{fa[0], fa[1], fa[2]}};
  const amrex::GpuArray<const Array4<const Real>, 3> a{
      {Array4<const Real>(aa[0]), Array4<const Real>(aa[1]), Array4<const Real>(aa[2])}};
  const amrex::GpuArray<Real, 3> dxa{{dx[0], dx[1], dx[2]}};
  hydro_umdrv(p->do_mol != 0, bx, geom, bclo, bchi, sarr, dsdt.array(), qarr, qauxar, srcqarr,
              dxa, dt, p->ppm_type, p->plm_iorder, p->use_pslope, p->use_flattening,
              p->transverse_reset_density, p->small, p->small_dens, p->small_pres, p->smallu,
              p->difmag, flx_arr, a, vol.array(), &pmap);
  const camr_flops::Counts c = camr_flops::counts();
  counts[0] = c.add;
  counts[1] = c.mul;
  counts[2] = c.div;
  counts[3] = c.sqrt;
  counts[4] = c.cmp;
  counts[5] = c.other;
  return amrex::shim_assert_count();
}
