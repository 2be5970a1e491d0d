// Shared pieces of the CPU oracle (test infrastructure): index layout, a small
// owning/non-owning Array4-style fab, the gamma-law EOS and the parameter
// defaults.  Everything here restates CAMR definitions; each item cites the
// reference line it follows.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <vector>

#include "oracle_abi.h"

namespace orc {

// Source/Utils/IndexDefines.H:17-89 (AMREX_SPACEDIM == 3, NUM_SPECIES = 3).
enum {
  URHO = 0, UMX = 1, UMY = 2, UMZ = 3, UEDEN = 4, UEINT = 5, UTEMP = 6,
  UFS = 7, NVAR = 10
};
enum {
  QRHO = 0, QU = 1, QV = 2, QW = 3, QGAME = 4, QPRES = 5, QREINT = 6,
  QTEMP = 7, QFS = 8, QVAR = 11
};
enum { QGAMC = 0, QC = 1, QCSML = 2, QDPDR = 3, QDPDE = 4, NQAUX = 5 };
enum { GDU = 1, GDV = 2, GDW = 3, GDPRES = 4, GDGAME = 5, NGDNV = 6 };
constexpr int NSPEC = 3;

// Source/EOS/PhysicsConstants.H:8-10.
constexpr double RU = 8.31446261815324e7;
constexpr double AIRMW = 26.93;

// Array4-style view, optionally owning its storage (filled with quiet NaN so
// that a read of a slot nothing wrote is visible in the results).
struct Fab {
  int lo[3] = {0, 0, 0};
  int hi[3] = {-1, -1, -1};
  int nc = 0;
  long long sj = 0, sk = 0, sn = 0;
  double* p = nullptr;
  std::vector<double> own;

  Fab() = default;
  Fab(const int l[3], const int h[3], int ncomp) { alloc(l, h, ncomp); }
  void alloc(const int l[3], const int h[3], int ncomp) {
    set_shape(l, h, ncomp);
    own.assign(size_t(sn) * nc, std::numeric_limits<double>::quiet_NaN());
    p = own.data();
  }
  void view(double* ptr, const int l[3], const int h[3], int ncomp) {
    set_shape(l, h, ncomp);
    p = ptr;
  }
  void set_shape(const int l[3], const int h[3], int ncomp) {
    for (int d = 0; d < 3; ++d) { lo[d] = l[d]; hi[d] = h[d]; }
    nc = ncomp;
    sj = hi[0] - lo[0] + 1;
    sk = sj * (hi[1] - lo[1] + 1);
    sn = sk * (hi[2] - lo[2] + 1);
  }
  double& operator()(int i, int j, int k, int n = 0) const {
    return p[(i - lo[0]) + (j - lo[1]) * sj + (k - lo[2]) * sk + n * sn];
  }
  bool contains(int i, int j, int k) const {
    return i >= lo[0] && i <= hi[0] && j >= lo[1] && j <= hi[1] &&
           k >= lo[2] && k <= hi[2];
  }
};

struct Box3 {
  int lo[3], hi[3];
};

inline Box3 grow(const Box3& b, int n) {
  Box3 r = b;
  for (int d = 0; d < 3; ++d) { r.lo[d] -= n; r.hi[d] += n; }
  return r;
}
inline Box3 grow(const Box3& b, int d, int n) {
  Box3 r = b; r.lo[d] -= n; r.hi[d] += n; return r;
}
// Faces normal to d of the cells of b (AMReX surroundingNodes(b, d)).
inline Box3 faces(const Box3& b, int d) {
  Box3 r = b; r.hi[d] += 1; return r;
}

template <class F>
inline void for_box(const Box3& b, F&& f) {
  for (int k = b.lo[2]; k <= b.hi[2]; ++k)
    for (int j = b.lo[1]; j <= b.hi[1]; ++j)
      for (int i = b.lo[0]; i <= b.hi[0]; ++i) f(i, j, k);
}

// Gamma-law EOS, Source/EOS/GammaLaw/EOS.H (gamma made a runtime value).
struct Eos {
  double gamma;
  // REY2P (:133-137): P = (gamma-1)*R*E
  double rey2p(double r, double e) const { return (gamma - 1.0) * r * e; }
  // EY2T (:115-122): T = (gamma-1)*E*wbar/RU
  double ey2t(double e) const {
    const double poverrho = (gamma - 1.0) * e;
    return poverrho * AIRMW / RU;
  }
  // RTY2E via T2Ei/TY2E (:24-31, :265-276): E = sum_n Y_n*Cv*T
  double rty2e(double t, const double* y) const {
    const double cv = RU / (AIRMW * (gamma - 1.0));
    double e = 0.0;
    for (int n = 0; n < NSPEC; ++n) e += y[n] * (cv * t);
    return e;
  }
};

inline void default_params(orc_params* p) {
  // Source/Params/_cpp_parameters
  p->do_mol = 0;
  p->ppm_type = 0;
  p->plm_iorder = 4;
  p->use_pslope = 0;
  p->use_flattening = 1;
  p->transverse_reset_density = 1;
  p->dual_energy_update_E_from_e = 1;
  p->allow_negative_energy = 0;
  p->allow_small_energy = 1;
  p->add_grav_src = 1;
  p->eb_weights_type = 2;  // :107
  p->riemann_solver = 0;
  p->difmag = 0.1;
  p->small = 1.e-8;
  p->small_dens = 1.e-7;
  p->small_temp = 1.e2;
  p->small_pres = 1.e-200;
  p->dual_energy_eta1 = 1.0e0;
  p->dual_energy_eta2 = 1.0e-4;
  p->const_grav = 0.0;
  p->cfl = 0.8;
  p->init_shrink = 1.0;
  p->change_max = 1.1;
  p->fixed_dt = -1.0;
  p->initial_dt = -1.0;
  p->max_dt = 1.e200;
  p->eos_gamma = 1.4;           // Source/EOS/GammaLaw/EOS.H:16
  p->smallu = 1.e-12;           // Source/Utils/CAMR_Constants.H:9
  p->small_num = 1.e-8;         // Source/Utils/CAMR_Constants.H:10
}

}  // namespace orc
