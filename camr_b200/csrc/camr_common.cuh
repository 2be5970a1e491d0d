// Shared device definitions: index layout, parameters, exact min/max, fab
// indexing.  Built with -fmad=false so that every product/sum rounds on its
// own, as the reference's CPU build (-ffp-contract=off) does.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "camr_b200.h"
#include "fastdiv.h"

namespace camr {

// Source/Utils/IndexDefines.H:17-89 (3-D, NUM_SPECIES = 3).
enum { URHO = 0, UMX = 1, UMY = 2, UMZ = 3, UEDEN = 4, UEINT = 5, UTEMP = 6, UFS = 7,
       NVAR = 10 };
enum { QRHO = 0, QU = 1, QV = 2, QW = 3, QGAME = 4, QPRES = 5, QREINT = 6, QTEMP = 7,
       QFS = 8, QVAR = 11 };
enum { QGAMC = 0, QC = 1, QCSML = 2, QDPDR = 3, QDPDE = 4, NQAUX = 5 };
enum { GDU = 1, GDV = 2, GDW = 3, GDPRES = 4, GDGAME = 5, NGDNV = 6 };
constexpr int NSPEC = 3;
constexpr int NGROW = 4;  // CAMR::numGrow() without EB (Source/CAMR.H:457-459)

// Source/EOS/PhysicsConstants.H:8-10.
constexpr double RU = 8.31446261815324e7;
constexpr double AIRMW = 26.93;

// std::max / std::min semantics (first argument wins ties and NaN
// comparisons), which the reference relies on; fmax/fmin differ on NaN and
// signed zero.
__host__ __device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }
__host__ __device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }

// Compact primitive record kept per cell (slots follow QVAR numbering for
// the ones the hydro reads; QGAME/QTEMP are never consumed downstream).
// Stored components of the q array, in this order:
enum { SQ_RHO = 0, SQ_U = 1, SQ_V = 2, SQ_W = 3, SQ_P = 4, SQ_REINT = 5, SQ_FS = 6,
       SQ_C = 9, SQ_CSML = 10, SQ_N = 11 };
// Edge-state record (normal predictor / transverse-corrected states):
enum { ES_RHO = 0, ES_U = 1, ES_V = 2, ES_W = 3, ES_P = 4, ES_REINT = 5, ES_FS = 6, ES_N = 9 };
// Flux record of the intermediate passes: the conserved fluxes the
// transverse corrections read, then the Riemann interface pressure and the
// interface velocity normal to the face (the only Riemann outputs read
// downstream: Godunov_utils_3D.H:114-117, :365-377).
enum { FR_RHO = 0, FR_MX = 1, FR_MY = 2, FR_MZ = 3, FR_E = 4, FR_FS = 5, FR_PRES = 8,
       FR_UN = 9, FR_N = 10 };

// Per-run constants handed to every kernel by value.
struct KParams {
  int ppm_type, plm_iorder, use_pslope, use_flattening, transverse_reset_density;
  int dual_energy_update_E_from_e, allow_negative_energy, allow_small_energy;
  int add_grav_src;
  int riemann_solver;  // 0 riemannus (the reference), 1 HLLC
  double difmag, small, small_dens, small_temp, small_pres, smallu, small_num;
  double dual_energy_eta1, dual_energy_eta2, const_grav, gamma;
};

inline KParams make_kparams(const camr_hydro_params& p) {
  KParams k;
  k.ppm_type = p.ppm_type;
  k.plm_iorder = p.plm_iorder;
  k.use_pslope = p.use_pslope;
  k.use_flattening = p.use_flattening;
  k.transverse_reset_density = p.transverse_reset_density;
  k.dual_energy_update_E_from_e = p.dual_energy_update_E_from_e;
  k.allow_negative_energy = p.allow_negative_energy;
  k.allow_small_energy = p.allow_small_energy;
  k.add_grav_src = p.add_grav_src;
  k.riemann_solver = p.riemann_solver;
  k.difmag = p.difmag;
  k.small = p.small;
  k.small_dens = p.small_dens;
  k.small_temp = p.small_temp;
  k.small_pres = p.small_pres;
  k.smallu = p.smallu;
  k.small_num = p.small_num;
  k.dual_energy_eta1 = p.dual_energy_eta1;
  k.dual_energy_eta2 = p.dual_energy_eta2;
  k.const_grav = p.const_grav;
  k.gamma = p.eos_gamma;
  return k;
}

// Geometry of the box being advanced and of its domain.
struct KGeom {
  int lo[3], hi[3];          // valid box bx
  int dlo[3], dhi[3];        // domain
  int bclo[3], bchi[3];
  double dx[3];
};

// Uniform index space shared by all intermediates of one box: the cells of
// grow(bx, NGROW) plus one more layer on the high side for faces.
struct Space {
  int lo[3];                 // bx.lo - NGROW
  int n[3];                  // bx extent + 2*NGROW + 1
  int64_t sy, sz, sn;
  __host__ __device__ int64_t idx(int i, int j, int k) const {
    return (i - lo[0]) + (j - lo[1]) * sy + (k - lo[2]) * sz;
  }
};

inline Space make_space(const int blo[3], const int bhi[3]) {
  Space s;
  for (int d = 0; d < 3; ++d) {
    s.lo[d] = blo[d] - NGROW;
    s.n[d] = bhi[d] - blo[d] + 1 + 2 * NGROW + 1;
  }
  s.sy = s.n[0];
  s.sz = s.sy * s.n[1];
  s.sn = s.sz * s.n[2];
  return s;
}

// Device view of a caller fab.
struct DFab {
  double* p;
  int lo[3];
  int64_t sy, sz, sn;
  __host__ __device__ double& operator()(int i, int j, int k, int n) const {
    return p[(i - lo[0]) + (j - lo[1]) * sy + (k - lo[2]) * sz + n * sn];
  }
};

inline DFab make_dfab(const camr_fab& f) {
  DFab d;
  d.p = f.ptr;
  for (int a = 0; a < 3; ++a) d.lo[a] = f.lo[a];
  d.sy = f.jstride;
  d.sz = f.kstride;
  d.sn = f.nstride;
  return d;
}

// A rectangular index region launched as a flat 1-D grid, i fastest.  Build
// it with make_region (a default-constructed one is empty).
struct Region {
  int lo[3] = {0, 0, 0}, n[3] = {0, 0, 0};
  Decode3 dc = {0, 0, 0, {0u, 0}, {0u, 0}};
  int64_t count() const { return int64_t(n[0]) * n[1] * n[2]; }
};

__device__ __forceinline__ bool region_cell(const Region& r, int64_t t, int& i, int& j, int& k) {
  if (t >= int64_t(r.n[0]) * r.n[1] * r.n[2]) return false;
  if (r.dc.fast) {
    decode3(r.dc, t, i, j, k);
  } else {
    // a region not built by make_region, or of 2^31 cells or more
    const int64_t nxy = int64_t(r.n[0]) * r.n[1];
    k = int(t / nxy);
    const int64_t rem = t - int64_t(k) * nxy;
    j = int(rem / r.n[0]);
    i = int(rem - int64_t(j) * r.n[0]);
  }
  i += r.lo[0];
  j += r.lo[1];
  k += r.lo[2];
  return true;
}

inline Region make_region(const int lo[3], const int hi[3]) {
  Region r;
  for (int d = 0; d < 3; ++d) {
    r.lo[d] = lo[d];
    r.n[d] = hi[d] - lo[d] + 1;
  }
  if (r.count() > 0) r.dc = make_decode3(r.n[0], r.n[1], r.n[2]);
  return r;
}

// Device error word: first failure wins.
struct DevError {
  int code;
  int i, j, k;
};

__device__ __forceinline__ void report_error(DevError* e, int code, int i, int j, int k) {
  if (e && atomicCAS(&e->code, 0, code) == 0) {
    e->i = i;
    e->j = j;
    e->k = k;
  }
}

void count_launch(int n = 1);
int64_t launches_now();        // kernels issued so far (camr_launch_count)
void launches_sub(int64_t n);  // take back launches counted during a capture
// CAMR_OK, or CAMR_ERR_CUDA with the CUDA error text kept for
// camr_last_error_string.
camr_status cuda_status_of(cudaError_t e);
const char* last_error_text();
// The parameter checks of the per-box hydro and the level drivers
// (Source/CAMR.cpp:160-190): CAMR_OK, or the status to return.
camr_status check_hydro_params(const camr_hydro_params* p);
// The library-wide device error word (camr_get_error) on the current
// device; looked up outside stream capture, cached for use inside it.
cudaError_t library_error_word(cudaStream_t st, DevError** out);

}  // namespace camr
