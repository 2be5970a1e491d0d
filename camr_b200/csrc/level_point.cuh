// Cell-level pieces of the level driver shared by the single-level and the
// two-level (AMR) drivers: the clean_state / computeTemp / FillPatch bodies,
// the fused end-of-step update, the CFL reduction and the dt control.
// Restated from Source/CAMR.cpp, Source/CAMR_advance.cpp and
// Source/Utils/CAMR_reset_internal_e.H (each function cites its lines).
#pragma once

#include <cuda_runtime.h>

#include <cfloat>

#include "hydro_kernels.cuh"

namespace camr {
namespace {

constexpr int kBlk = 256;
// resident 256-thread blocks per SM asked of the end-of-step update kernels:
// with 3 (at most 85 registers) the 256^3 CTU update took 1.98 ms against
// 2.68 ms with 4 (64 registers, spills) and 3.20 ms uncapped (76 registers)
#ifndef CAMR_MINB_UPDATE
#define CAMR_MINB_UPDATE 3
#endif
inline unsigned grid_of(int64_t n) { return unsigned((n + kBlk - 1) / kBlk); }
__device__ __forceinline__ int64_t tid() { return int64_t(blockIdx.x) * blockDim.x + threadIdx.x; }

// Per-level constants of the state arrays (padded domain, NVAR comps).
struct LGeom {
  int dlo[3], dhi[3];       // domain
  int plo[3];               // padded lo = dlo - NGROW
  int pn[3];                // padded extent
  int64_t sy, sz, sn;
  int periodic[3];
  int bclo[3], bchi[3];
  int boxsz[3];             // enforce_min_density window (box size)
  double dx[3];
  // flat-index decoding of valid / padded cells (lgeom_finish; without it
  // the kernels divide in 64 bits)
  Decode3 vdc = {0, 0, 0, {0u, 0}, {0u, 0}};
  Decode3 pdc = {0, 0, 0, {0u, 0}, {0u, 0}};
  __host__ __device__ int64_t idx(int i, int j, int k) const {
    return (i - plo[0]) + (j - plo[1]) * sy + (k - plo[2]) * sz;
  }
};

// Call once the domain and padded extents are set.
inline void lgeom_finish(LGeom& L) {
  L.vdc = make_decode3(L.dhi[0] - L.dlo[0] + 1, L.dhi[1] - L.dlo[1] + 1, L.dhi[2] - L.dlo[2] + 1);
  L.pdc = make_decode3(L.pn[0], L.pn[1], L.pn[2]);
}

struct LevelState {
  double* S;       // state (valid cells meaningful)
  double* S_old;
  double* B;       // Sborder
  double* B2;      // MOL stage-2 Sborder
  double* flx[3];  // face fluxes of the domain box (NVAR comps, Space-indexed)
  double* work;
  Work w;
  double* dt_cur;          // device: dt of the step being taken
  double* dt_hist;         // device: dt of every step
  unsigned long long* dtmin_bits;  // device: running CFL min
  int* nstep;              // device: steps taken
  DevError* err;
};

// BC kind of component n in direction dir for physical BC word phys
// (Source/Utils/CAMR_setup.cpp:19-21): 1 ext_dir, 2 foextrap,
// 3 reflect_even, 4 reflect_odd.
__device__ __forceinline__ int bc_kind(int n, int dir, int phys) {
  const int scalar_bc[6] = {0, 1, 2, 3, 3, 3};
  const int norm_vel_bc[6] = {0, 1, 2, 4, 4, 4};
  const int tang_vel_bc[6] = {0, 1, 2, 3, 3, 4};
  if (n >= UMX && n <= UMZ) return (n - UMX == dir) ? norm_vel_bc[phys] : tang_vel_bc[phys];
  return scalar_bc[phys];
}

// computeTemp body: reset_internal_energy (Source/Utils/CAMR_reset_internal_e.H:13-129)
// then T (Source/CAMR.cpp:1166-1183).
__device__ __forceinline__ void compute_temp(double* s, const KParams& P) {
  const double rho = s[URHO];
  const double rhoInv = 1.0 / rho;
  const double Up = s[UMX] * rhoInv;
  const double Vp = s[UMY] * rhoInv;
  const double Wp = s[UMZ] * rhoInv;
  const double ke = 0.5 * (Up * Up + Vp * Vp + Wp * Wp);
  const double eden = s[UEDEN] * rhoInv;
  double massfrac[NSPEC];
#pragma unroll
  for (int sp = 0; sp < NSPEC; ++sp) massfrac[sp] = s[sp + UFS] * rhoInv;
  double e_out = 0.;
  double small_e = 0.;
  const double small_T = P.small_temp;
  if (P.allow_small_energy == 0) {
    small_e = eos_rty2e(P.gamma, small_T, massfrac);
    if (eden < small_e) {
      if (s[UEINT] * rhoInv < small_e) {
        const double T = dmax(s[UTEMP], small_T);
        e_out = eos_rty2e(P.gamma, T, massfrac);
        s[UEINT] = rho * e_out;
      }
      s[UEDEN] = s[UEINT] + rho * ke;
    } else {
      const double rho_eint = s[UEDEN] - s[URHO] * ke;
      if (rho_eint > 0. && rho_eint / s[UEDEN] > P.dual_energy_eta2) s[UEINT] = rho_eint;
      if (s[UEINT] * rhoInv < small_e) {
        const double T = dmax(s[UTEMP], small_T);
        e_out = eos_rty2e(P.gamma, T, massfrac);
        if (P.dual_energy_update_E_from_e == 1) s[UEDEN] += (rho * e_out - s[UEINT]);
        s[UEINT] = s[URHO] * e_out;
      }
    }
  } else if (P.allow_negative_energy == 0) {
    if (s[UEDEN] < 0.) {
      if (s[UEINT] < 0.) {
        e_out = eos_rty2e(P.gamma, small_T, massfrac);
        s[UEINT] = rho * e_out;
      }
      s[UEDEN] = s[UEINT] + rho * ke;
    } else {
      const double rho_eint = s[UEDEN] - rho * ke;
      if (rho_eint > 0. && rho_eint / s[UEDEN] > P.dual_energy_eta2) {
        s[UEINT] = rho_eint;
      } else if (s[UEINT] > 0 && P.dual_energy_update_E_from_e == 1) {
        s[UEDEN] = s[UEINT] + rho * ke;
      } else if (s[UEINT] <= 0.) {
        e_out = eos_rty2e(P.gamma, small_T, massfrac);
        s[UEINT] = rho * e_out;
        if (P.dual_energy_update_E_from_e == 1) s[UEDEN] += (rho * e_out - s[UEINT]);
      }
    }
  } else {
    s[UEINT] = s[UEDEN] - rho * ke;
  }
  const double rhoInv2 = 1.0 / s[URHO];
  const double e = s[UEINT] * rhoInv2;
  s[UTEMP] = eos_ey2t(P.gamma, e);
}

// normalize_species (Source/CAMR.cpp:884-905).
__device__ __forceinline__ void normalize_species(double* s) {
  double sum = 0.;
#pragma unroll
  for (int sp = 0; sp < NSPEC; ++sp) {
    s[UFS + sp] = dmax(dmin(s[URHO], s[UFS + sp]), 0.0);
    sum += s[UFS + sp];
  }
  if (s[URHO] > 0.) {
    sum /= s[URHO];
#pragma unroll
    for (int sp = 0; sp < NSPEC; ++sp) s[UFS + sp] /= sum;
  }
}

__device__ __forceinline__ void load_cell(const double* a, const LGeom& L, int64_t at, double* s) {
#pragma unroll
  for (int n = 0; n < NVAR; ++n) s[n] = a[at + n * L.sn];
}
__device__ __forceinline__ void store_cell(double* a, const LGeom& L, int64_t at, const double* s) {
#pragma unroll
  for (int n = 0; n < NVAR; ++n) a[at + n * L.sn] = s[n];
}

// enforce_min_density (Source/CAMR.cpp:941-1045) of the valid cell (i,j,k)
// reading neighbours from `src` (the array being cleaned, before cleaning),
// within the level box that contains the cell.
__device__ void enforce_min_density(double* s, const double* src, const LGeom& L,
                                    const KParams& P, int i, int j, int k, DevError* err) {
  if (s[URHO] == 0.) {
    report_error(err, 3, i, j, k);
    return;
  }
  if (!(s[URHO] < P.small_dens)) return;
  int blo[3], bhi[3];
  const int c[3] = {i, j, k};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int b = (c[d] - L.dlo[d]) / L.boxsz[d];
    blo[d] = L.dlo[d] + b * L.boxsz[d];
    bhi[d] = min(blo[d] + L.boxsz[d] - 1, L.dhi[d]);
  }
  double max_dens = s[URHO];
  int is = i, js = j, ks = k;
  for (int kk = -1; kk <= 1; kk++)
    for (int jj = -1; jj <= 1; jj++)
      for (int ii = -1; ii <= 1; ii++) {
        if (i + ii >= blo[0] && j + jj >= blo[1] && k + kk >= blo[2] && i + ii <= bhi[0] &&
            j + jj <= bhi[1] && k + kk <= bhi[2]) {
          const double r = src[L.idx(i + ii, j + jj, k + kk)];
          if (r > max_dens) {
            is = i + ii; js = j + jj; ks = k + kk;
            max_dens = r;
          }
        }
      }
  if (max_dens < P.small_dens) {
    double massfrac[NSPEC];
#pragma unroll
    for (int sp = 0; sp < NSPEC; ++sp) massfrac[sp] = s[UFS + sp] / s[URHO];
    const double small_e = eos_rty2e(P.gamma, P.small_temp, massfrac);
    s[URHO] = P.small_dens;
    s[UTEMP] = P.small_temp;
    s[UMX] = 0.;
    s[UMY] = 0.;
    s[UMZ] = 0.;
    s[UEINT] = P.small_dens * small_e;
    s[UEDEN] = s[UEINT];
  } else {
    load_cell(src, L, L.idx(is, js, ks), s);
  }
}

__device__ __forceinline__ bool padded_cell(const LGeom& L, int64_t t, int& i, int& j, int& k) {
  const int64_t n = int64_t(L.pn[0]) * L.pn[1] * L.pn[2];
  if (t >= n) return false;
  if (L.pdc.fast) {
    decode3(L.pdc, t, i, j, k);
  } else {
    const int64_t nxy = int64_t(L.pn[0]) * L.pn[1];
    k = int(t / nxy);
    const int64_t r = t - int64_t(k) * nxy;
    j = int(r / L.pn[0]);
    i = int(r - int64_t(j) * L.pn[0]);
  }
  i += L.plo[0];
  j += L.plo[1];
  k += L.plo[2];
  return true;
}

__device__ __forceinline__ bool valid_cell(const LGeom& L, int64_t t, int& i, int& j, int& k) {
  const int n0 = L.dhi[0] - L.dlo[0] + 1, n1 = L.dhi[1] - L.dlo[1] + 1,
            n2 = L.dhi[2] - L.dlo[2] + 1;
  if (t >= int64_t(n0) * n1 * n2) return false;
  if (L.vdc.fast) {
    decode3(L.vdc, t, i, j, k);
  } else {
    const int64_t nxy = int64_t(n0) * n1;
    k = int(t / nxy);
    const int64_t r = t - int64_t(k) * nxy;
    j = int(r / n0);
    i = int(r - int64_t(j) * n0);
  }
  i += L.dlo[0];
  j += L.dlo[1];
  k += L.dlo[2];
  return true;
}

// Cells below the density floor met by a fused clean or update pass.  The
// reference's enforce_min_density (Source/CAMR.cpp:941-1045) walks a box's
// cells in raster order and resets each one in place, so a cell reset early
// can be the neighbour a later cell copies: a parallel pass cannot
// reproduce that.  The pass therefore appends such cells here and
// k_floor_fixup redoes them one after another in the reference's order.
// count == nullptr: no list; the pass then resets from the neighbours'
// values before the reset (exact when no two flagged cells are neighbours)
// and an update pass reports the crossing in the error word.
constexpr int kFloorCap = 16384;
// The fixups sort the list in dynamic shared memory (above the 48 KB
// default: floor_prepare / kf_floor_prepare raise each kernel's limit).
constexpr size_t kFloorSmem = sizeof(int64_t) * kFloorCap;
struct FloorList {
  int* count = nullptr;        // cells appended by the current pass (reset by the fixup)
  int64_t* cells = nullptr;    // their padded-array indices (kFloorCap)
  double* enforced = nullptr;  // kFloorCap x NVAR scratch of the fixup
  unsigned long long* total = nullptr;  // cells reset since the level was created
};

__device__ __forceinline__ void floor_push(const FloorList& fl, int64_t at) {
  const int slot = atomicAdd(fl.count, 1);
  if (slot < kFloorCap) fl.cells[slot] = at;
}

// clean_state on valid cells: S_old = clean(S)  (CAMR_advance.cpp:83).
__global__ void __launch_bounds__(kBlk) k_clean_copy(LGeom L, KParams P, const double* S,
                                                      double* out, DevError* err,
                                                      FloorList fl = FloorList{}) {
  int i, j, k;
  if (!valid_cell(L, tid(), i, j, k)) return;
  const int64_t at = L.idx(i, j, k);
  double s[NVAR];
  load_cell(S, L, at, s);
  if (fl.count && s[URHO] < P.small_dens) floor_push(fl, at);
  enforce_min_density(s, S, L, P, i, j, k, err);
  normalize_species(s);
  compute_temp(s, P);
  store_cell(out, L, at, s);
}

// expand_state: FillPatch(src) into B, then clean_state(B)
// (Source/CAMR.cpp:1243-1262).  Cells inside the periodic extension of the
// domain take the cleaned value of their periodic image (FillBoundary after
// normalize_species); physical-boundary ghosts take the BC-mapped values of
// src (foextrap / reflect_even / reflect_odd; ext_dir copies the boundary
// cell as Exec/Sod's bcnormal does) and only computeTemp.
__global__ void __launch_bounds__(kBlk) k_expand(LGeom L, KParams P, const double* src,
                                                  double* B, DevError* err,
                                                  FloorList fl = FloorList{}) {
  int i, j, k;
  if (!padded_cell(L, tid(), i, j, k)) return;
  const int c[3] = {i, j, k};
  int img[3];
  bool physical = false;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    img[d] = c[d];
    if (c[d] < L.dlo[d] || c[d] > L.dhi[d]) {
      if (L.periodic[d]) {
        const int len = L.dhi[d] - L.dlo[d] + 1;
        img[d] = L.dlo[d] + (((c[d] - L.dlo[d]) % len) + len) % len;
      } else {
        physical = true;
      }
    }
  }
  double s[NVAR];
  if (!physical) {
    load_cell(src, L, L.idx(img[0], img[1], img[2]), s);
    // the valid cell itself (not a periodic ghost image) joins the list
    if (fl.count && s[URHO] < P.small_dens && img[0] == i && img[1] == j && img[2] == k)
      floor_push(fl, L.idx(i, j, k));
    enforce_min_density(s, src, L, P, img[0], img[1], img[2], err);
    normalize_species(s);
  } else {
#pragma unroll
    for (int n = 0; n < NVAR; ++n) {
      int id[3] = {img[0], img[1], img[2]};
      bool neg = false;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        if (L.periodic[d]) continue;
        if (id[d] < L.dlo[d]) {
          const int t = bc_kind(n, d, L.bclo[d]);
          if (t == 1 || t == 2) id[d] = L.dlo[d];
          else { id[d] = 2 * L.dlo[d] - id[d] - 1; if (t == 4) neg = !neg; }
        } else if (id[d] > L.dhi[d]) {
          const int t = bc_kind(n, d, L.bchi[d]);
          if (t == 1 || t == 2) id[d] = L.dhi[d];
          else { id[d] = 2 * L.dhi[d] - id[d] + 1; if (t == 4) neg = !neg; }
        }
      }
      const double v = src[L.idx(id[0], id[1], id[2]) + n * L.sn];
      s[n] = neg ? -v : v;
    }
  }
  compute_temp(s, P);
  store_cell(B, L, L.idx(i, j, k), s);
}

// sources_for_hydro of a CTU step with gravity (Source/Hydro/
// CAMR_construct_hydro_source.cpp:28-34): zero, plus 1.0 x the old-time
// gravity source (Source/GravitySrc.cpp:36-70, from the cleaned S_old) on
// valid cells, copied to the ghost cells inside the periodic extension of
// the domain (FillBoundary); ghost cells beyond a physical boundary keep 0.
__global__ void __launch_bounds__(kBlk) k_src_hydro(LGeom L, KParams P, const double* S_old,
                                                     double* out) {
  int i, j, k;
  if (!padded_cell(L, tid(), i, j, k)) return;
  const int c[3] = {i, j, k};
  int img[3];
  bool physical = false;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    img[d] = c[d];
    if (c[d] < L.dlo[d] || c[d] > L.dhi[d]) {
      if (L.periodic[d]) {
        const int len = L.dhi[d] - L.dlo[d] + 1;
        img[d] = L.dlo[d] + (((c[d] - L.dlo[d]) % len) + len) % len;
      } else {
        physical = true;
      }
    }
  }
  const int64_t at = L.idx(i, j, k);
  double src[NVAR];
#pragma unroll
  for (int n = 0; n < NVAR; ++n) src[n] = 0.0;
  if (!physical) {
    const int64_t im = L.idx(img[0], img[1], img[2]);
    src[UMZ] = P.const_grav * S_old[im + URHO * L.sn];
    src[UEDEN] = P.const_grav * S_old[im + UMZ * L.sn];
#pragma unroll
    for (int n = 0; n < NVAR; ++n) out[at + n * L.sn] = 0.0 + 1.0 * src[n];
  } else {
#pragma unroll
    for (int n = 0; n < NVAR; ++n) out[at + n * L.sn] = 0.0;
  }
}

// Block-wide min of positive doubles into *bits (order-preserving as u64).
__device__ __forceinline__ void block_min_dt(double v, unsigned long long* bits) {
  unsigned long long b = __double_as_longlong(v);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long other = __shfl_down_sync(0xffffffffu, b, o);
    b = (other < b) ? other : b;
  }
  __shared__ unsigned long long warp_min[kBlk / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) warp_min[wid] = b;
  __syncthreads();
  if (wid == 0) {
    b = (lane < kBlk / 32) ? warp_min[lane] : ~0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long other = __shfl_down_sync(0xffffffffu, b, o);
      b = (other < b) ? other : b;
    }
    if (lane == 0) atomicMin(bits, b);
  }
}

// CAMR_estdt_hydro body (Source/Utils/Timestep.H:34-56) of one cell.
__device__ __forceinline__ double cell_dt(const double* s, const LGeom& L, const KParams& P) {
  const double rho = s[URHO];
  const double rhoInv = 1.0 / rho;
  const double eint = s[UEINT] / rho;
  const double pres = (P.gamma - 1.0) * rho * eint;
  const double c = sqrt(P.gamma * pres / rho);
  double dt = DBL_MAX;
  const double ux = s[UMX] * rhoInv;
  dt = dmin(dt, L.dx[0] / (c + fabs(ux)));
  const double uy = s[UMY] * rhoInv;
  dt = dmin(dt, L.dx[1] / (c + fabs(uy)));
  const double uz = s[UMZ] * rhoInv;
  dt = dmin(dt, L.dx[2] / (c + fabs(uz)));
  return dt;
}

__global__ void __launch_bounds__(kBlk) k_est_dt(LGeom L, KParams P, const double* S,
                                                  unsigned long long* bits) {
  int i, j, k;
  double v = DBL_MAX;
  if (valid_cell(L, tid(), i, j, k)) {
    double s[NVAR];
    load_cell(S, L, L.idx(i, j, k), s);
    v = cell_dt(s, L, P);
  }
  block_min_dt(v, bits);
}

// Error code of a density that fails `rho >= small_dens`: 3 exactly zero
// (amrex::Error in enforce_min_density), 5 below the floor, 2 NaN.
__device__ __forceinline__ int floor_code(double rho, const KParams& P) {
  return rho == 0. ? 3 : (rho < P.small_dens ? 5 : 2);
}

// The end of a level step on one valid cell, from the state right after
// the hydro Saxpy: clean_state, the new-source correction (+ its
// clean_state) and, with `post`, post_timestep's clean_state (a level that
// has a finer level above it cleans after reflux and average-down instead);
// then the cell's CFL dt.
__device__ __forceinline__ double finish_step(double* s, const double* sold, const KParams& P,
                                              const LGeom& L, double dt, int i, int j, int k,
                                              DevError* err, bool post = true) {
  // clean_state(S_new).  The density floor is handled before this point
  // (k_floor_fixup resets the cells below it); a density still below the
  // floor here (no floor list) or NaN is reported in the error word.
  if (!(s[URHO] >= P.small_dens)) report_error(err, floor_code(s[URHO], P), i, j, k);
  normalize_species(s);
  compute_temp(s, P);
  if (P.add_grav_src) {
    double src[NVAR];
#pragma unroll
    for (int n = 0; n < NVAR; ++n) src[n] = 0.0;
    src[UMZ] = 0.5 * P.const_grav * (s[URHO] - sold[URHO]);
    src[UEDEN] = 0.5 * P.const_grav * (s[UMZ] - sold[UMZ]);
#pragma unroll
    for (int n = 0; n < NVAR; ++n) s[n] += dt * src[n];
    if (!(s[URHO] >= P.small_dens)) report_error(err, floor_code(s[URHO], P), i, j, k);
    normalize_species(s);
    compute_temp(s, P);
  }
  if (post) {
    if (!(s[URHO] >= P.small_dens)) report_error(err, floor_code(s[URHO], P), i, j, k);
    normalize_species(s);
    compute_temp(s, P);
  }
  return cell_dt(s, L, P);
}

// hydro_update of one cell (Hydro_utils_K.H:239-257): returns dSdt.
__device__ __forceinline__ void cell_dsdt(const LGeom& L, const Space& sp, int i, int j, int k,
                                          double* const* flx, double* const* qf, double* hs) {
  const double a0 = L.dx[1] * L.dx[2], a1 = L.dx[0] * L.dx[2], a2 = L.dx[0] * L.dx[1];
  const double vol = L.dx[0] * L.dx[1] * L.dx[2];
  const int64_t at = sp.idx(i, j, k);
  const int64_t sn = sp.sn;
  const double* q1 = qf[0];
  const double* q2 = qf[1];
  const double* q3 = qf[2];
  const double pdivu =
      0.5 *
      ((q1[at + 1] + q1[at]) * (q1[at + 1 + sn] * a0 - q1[at + sn] * a0) +
       (q2[at + sp.sy] + q2[at]) * (q2[at + sp.sy + sn] * a1 - q2[at + sn] * a1) +
       (q3[at + sp.sz] + q3[at]) * (q3[at + sp.sz + sn] * a2 - q3[at + sn] * a2)) /
      vol;
  const double volinv = 1.0 / vol;
  const double* fx = flx[0];
  const double* fy = flx[1];
  const double* fz = flx[2];
#pragma unroll
  for (int n = 0; n < NVAR; ++n) {
    const int64_t o = at + n * sn;
    // construct_hydro_source zeroes src_to_fill first (:14): 0 + update.
    hs[n] = 0.0 + (fx[o] - fx[o + 1] + fy[o] - fy[o + sp.sy] + fz[o] - fz[o + sp.sz]) * volinv;
  }
  hs[UEINT] -= pdivu;
}

struct FluxPtrs {
  double* f[3];
  double* q[3];
};

// CTU: the state right after the Saxpys, S_new = Sborder (+ dt*src_old) +
// dt*dSdt; sold receives the old density and z momentum the gravity terms
// read (zero without gravity).
__device__ __forceinline__ void ctu_raw(const LGeom& L, const Space& sp, const KParams& P,
                                        double dt, const double* B, const double* S_old,
                                        const FluxPtrs& fp, int i, int j, int k, double* s,
                                        double* sold) {
  const int64_t at = L.idx(i, j, k);
  double hs[NVAR];
  load_cell(B, L, at, s);
#pragma unroll
  for (int n = 0; n < NVAR; ++n) sold[n] = 0.0;
  if (P.add_grav_src) {
    sold[URHO] = S_old[at + URHO * L.sn];
    sold[UMZ] = S_old[at + UMZ * L.sn];
  }
  if (P.add_grav_src) {
    double src[NVAR];
#pragma unroll
    for (int n = 0; n < NVAR; ++n) src[n] = 0.0;
    src[UMZ] = P.const_grav * sold[URHO];
    src[UEDEN] = P.const_grav * sold[UMZ];
#pragma unroll
    for (int n = 0; n < NVAR; ++n) s[n] += dt * src[n];
  }
  cell_dsdt(L, sp, i, j, k, fp.f, fp.q, hs);
#pragma unroll
  for (int n = 0; n < NVAR; ++n) s[n] += dt * hs[n];
}

// CTU: S_new = Sborder (+ dt*src_old) + dt*dSdt, then finish_step.  With a
// floor list, a cell below the density floor keeps its post-Saxpy state
// and joins the list (k_floor_fixup finishes it).
__global__ void __launch_bounds__(kBlk, CAMR_MINB_UPDATE) k_update_ctu(LGeom L, Space sp, KParams P,
                                                      const double* dtp, const double* B,
                                                      const double* S_old, FluxPtrs fp,
                                                      double* S, unsigned long long* bits,
                                                      DevError* err, int post = 1,
                                                      FloorList fl = FloorList{}) {
  int i, j, k;
  double v = DBL_MAX;
  if (valid_cell(L, tid(), i, j, k)) {
    const double dt = *dtp;
    const int64_t at = L.idx(i, j, k);
    double s[NVAR], sold[NVAR];
    ctu_raw(L, sp, P, dt, B, S_old, fp, i, j, k, s, sold);
    if (fl.count && s[URHO] < P.small_dens) {
      floor_push(fl, at);
    } else {
      v = finish_step(s, sold, P, L, dt, i, j, k, err, post != 0);
    }
    store_cell(S, L, at, s);
  }
  if (bits) block_min_dt(v, bits);
}

// MOL stage 1: S_new = Sborder (+ dt*src_old) + dt*k1 (not cleaned).
__global__ void __launch_bounds__(kBlk) k_update_mol1(LGeom L, Space sp, KParams P,
                                                       const double* dtp, const double* B,
                                                       const double* S_old, FluxPtrs fp,
                                                       double* S) {
  int i, j, k;
  if (!valid_cell(L, tid(), i, j, k)) return;
  const double dt = *dtp;
  const int64_t at = L.idx(i, j, k);
  double s[NVAR], hs[NVAR];
  load_cell(B, L, at, s);
  if (P.add_grav_src) {
    double src[NVAR];
#pragma unroll
    for (int n = 0; n < NVAR; ++n) src[n] = 0.0;
    src[UMZ] = P.const_grav * S_old[at + URHO * L.sn];
    src[UEDEN] = P.const_grav * S_old[at + UMZ * L.sn];
#pragma unroll
    for (int n = 0; n < NVAR; ++n) s[n] += dt * src[n];
  }
  cell_dsdt(L, sp, i, j, k, fp.f, fp.q, hs);
#pragma unroll
  for (int n = 0; n < NVAR; ++n) s[n] += dt * hs[n];
  store_cell(S, L, at, s);
}

// MOL stage 2 right after the LinComb and Saxpy (CAMR_advance.cpp:134-135):
// S_new = 0.5*Sborder2 + 0.5*S_old + 0.5*dt*k2; sold = S_old.
__device__ __forceinline__ void mol2_raw(const LGeom& L, const Space& sp, double dt,
                                         const double* B2, const double* S_old,
                                         const FluxPtrs& fp, int i, int j, int k, double* s,
                                         double* sold) {
  const int64_t at = L.idx(i, j, k);
  double b[NVAR], hs[NVAR];
  load_cell(B2, L, at, b);
  load_cell(S_old, L, at, sold);
#pragma unroll
  for (int n = 0; n < NVAR; ++n) s[n] = 0.5 * b[n] + 0.5 * sold[n];
  cell_dsdt(L, sp, i, j, k, fp.f, fp.q, hs);
#pragma unroll
  for (int n = 0; n < NVAR; ++n) s[n] += 0.5 * dt * hs[n];
}

// MOL stage 2, then finish_step (floor list as k_update_ctu).
__global__ void __launch_bounds__(kBlk, CAMR_MINB_UPDATE) k_update_mol2(LGeom L, Space sp, KParams P,
                                                       const double* dtp, const double* B2,
                                                       const double* S_old, FluxPtrs fp,
                                                       double* S, unsigned long long* bits,
                                                       DevError* err, int post = 1,
                                                       FloorList fl = FloorList{}) {
  int i, j, k;
  double v = DBL_MAX;
  if (valid_cell(L, tid(), i, j, k)) {
    const double dt = *dtp;
    const int64_t at = L.idx(i, j, k);
    double s[NVAR], sold[NVAR];
    mol2_raw(L, sp, dt, B2, S_old, fp, i, j, k, s, sold);
    if (fl.count && s[URHO] < P.small_dens) {
      floor_push(fl, at);
    } else {
      v = finish_step(s, sold, P, L, dt, i, j, k, err, post != 0);
    }
    store_cell(S, L, at, s);
  }
  if (bits) block_min_dt(v, bits);
}

// What k_floor_fixup finishes: the pass whose list it reads.  The DSDT
// modes are the updates of a level whose hydro right-hand side is an array
// (the EB level): CTU S_new = Sborder (+ dt*src_old) + dt*dsdt, MOL stage 2
// S_new = 0.5*Sborder2 + 0.5*S_old + 0.5*dt*dsdt.
// INPLACE: a pass that left the raw state in the array (in == out) for a
// later kernel to finish.
enum { FLOOR_CLEAN = 0, FLOOR_EXPAND = 1, FLOOR_CTU = 2, FLOOR_MOL2 = 3, FLOOR_DSDT_CTU = 4,
       FLOOR_DSDT_MOL2 = 5, FLOOR_INPLACE = 6 };

struct FloorArgs {
  const double* in;   // CLEAN / EXPAND: the array being cleaned
  double* out;        // CLEAN: S_old; EXPAND: Sborder; CTU / MOL2: S_new
  const double* B;    // CTU: Sborder; MOL2: Sborder2
  const double* S_old;
  FluxPtrs fp;
  Space sp;
  const double* dtp;
  unsigned long long* bits;  // CFL minimum (CTU / MOL2; may be null)
  int post;
  const double* dsdt = nullptr;  // DSDT modes: the hydro right-hand side
};

// The DSDT modes' post-Saxpy state of a cell (the operations of the EB
// level's update kernels).
template <int MODE>
__device__ __forceinline__ void dsdt_raw(const LGeom& L, const KParams& P, const FloorArgs& a,
                                         int64_t at, double* s) {
  const double dt = *a.dtp;
  if constexpr (MODE == FLOOR_DSDT_CTU) {
    load_cell(a.B, L, at, s);
    if (P.add_grav_src) {
      double src[NVAR];
#pragma unroll
      for (int n = 0; n < NVAR; ++n) src[n] = 0.0;
      src[UMZ] = P.const_grav * a.S_old[at + URHO * L.sn];
      src[UEDEN] = P.const_grav * a.S_old[at + UMZ * L.sn];
#pragma unroll
      for (int n = 0; n < NVAR; ++n) s[n] += dt * src[n];
    }
#pragma unroll
    for (int n = 0; n < NVAR; ++n) s[n] += dt * a.dsdt[at + n * L.sn];
  } else {
    double b[NVAR], sold[NVAR];
    load_cell(a.B, L, at, b);
    load_cell(a.S_old, L, at, sold);
#pragma unroll
    for (int n = 0; n < NVAR; ++n) s[n] = 0.5 * b[n] + 0.5 * sold[n];
#pragma unroll
    for (int n = 0; n < NVAR; ++n) s[n] += 0.5 * dt * a.dsdt[at + n * L.sn];
  }
}

// Sort key of a listed cell: its level box, then its padded index (raster
// order inside the box).
__device__ __forceinline__ int64_t floor_key(const LGeom& L, int64_t at, int i, int j, int k) {
  const int nb0 = (L.dhi[0] - L.dlo[0] + L.boxsz[0]) / L.boxsz[0];
  const int nb1 = (L.dhi[1] - L.dlo[1] + L.boxsz[1]) / L.boxsz[1];
  const int64_t box = (i - L.dlo[0]) / L.boxsz[0] +
                      int64_t(nb0) * ((j - L.dlo[1]) / L.boxsz[1] +
                                      int64_t(nb1) * ((k - L.dlo[2]) / L.boxsz[2]));
  return (box << 40) | at;
}

__device__ __forceinline__ int floor_find(const int64_t* key, int n, int64_t want) {
  int lo = 0, hi = n - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    if (key[mid] == want) return mid;
    if (key[mid] < want) lo = mid + 1;
    else hi = mid - 1;
  }
  return -1;
}

__device__ __forceinline__ void decode_cell(const LGeom& L, int64_t at, int& i, int& j, int& k) {
  k = int(at / L.sz);
  const int64_t r = at - int64_t(k) * L.sz;
  j = int(r / L.sy);
  i = int(r - int64_t(j) * L.sy);
  i += L.plo[0];
  j += L.plo[1];
  k += L.plo[2];
}

// The state of a cell as enforce_min_density finds it before any reset:
// the array being cleaned, or (updates) the post-Saxpy state, which the
// update pass stored for listed cells and which is recomputed for others.
template <int MODE>
__device__ __forceinline__ void floor_raw(const LGeom& L, const KParams& P, const FloorArgs& a,
                                          bool listed, int64_t at, int i, int j, int k,
                                          double* s) {
  if constexpr (MODE == FLOOR_CLEAN || MODE == FLOOR_EXPAND || MODE == FLOOR_INPLACE) {
    load_cell(a.in, L, at, s);
  } else {
    if (listed) {
      load_cell(a.out, L, at, s);
    } else if constexpr (MODE == FLOOR_DSDT_CTU || MODE == FLOOR_DSDT_MOL2) {
      dsdt_raw<MODE>(L, P, a, at, s);
    } else {
      double sold[NVAR];
      if constexpr (MODE == FLOOR_CTU) ctu_raw(L, a.sp, P, *a.dtp, a.B, a.S_old, a.fp, i, j, k, s, sold);
      else mol2_raw(L, a.sp, *a.dtp, a.B, a.S_old, a.fp, i, j, k, s, sold);
    }
  }
}

// Sort n listed keys (box << 40 | array index) in shared memory, ascending:
// bitonic over the next power of two, padded with INT64_MAX.  All threads
// of the block call it.
__device__ __forceinline__ void floor_sort(int64_t* key, int n) {
  int N = 1;
  while (N < n) N <<= 1;
  for (int t = threadIdx.x; t < N; t += blockDim.x)
    if (t >= n) key[t] = INT64_MAX;
  __syncthreads();
  for (int size = 2; size <= N; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int t = threadIdx.x; t < N; t += blockDim.x) {
        const int u = t ^ stride;
        if (u > t) {
          const bool up = (t & size) == 0;
          const int64_t x = key[t], y = key[u];
          if ((x > y) == up) {
            key[t] = y;
            key[u] = x;
          }
        }
      }
      __syncthreads();
    }
  }
}

constexpr int64_t kFloorAtMask = (int64_t(1) << 40) - 1;

// enforce_min_density (Source/CAMR.cpp:941-1045) on the sorted listed
// cells in the reference's order -- box by box, cells in raster order, each
// reset kept in `enf` so that later cells of the box see it; one thread per
// box (a cell's window never leaves its box, so boxes are independent).
// The policy gives the pass's view of the level:
//   decode(box, at, i, j, k)         cell of an array index
//   window(box, i, j, k, blo, bhi)   enforce_min_density's window (the box)
//   idx(box, i, j, k)                array index of a cell
//   dens(box, at)                    density as the pass left it
//   raw(listed, box, at, i, j, k, s) the state enforce_min_density sees
template <class Pol>
__device__ __forceinline__ void floor_walk(const Pol& pol, const KParams& P, const int64_t* key,
                                           int n, double* enf, DevError* err) {
  for (int t0 = threadIdx.x; t0 < n; t0 += blockDim.x) {
    const int64_t box = key[t0] >> 40;
    if (t0 > 0 && (key[t0 - 1] >> 40) == box) continue;  // not the first cell of its box
    for (int m = t0; m < n && (key[m] >> 40) == box; ++m) {
      const int64_t at = key[m] & kFloorAtMask;
      int i, j, k;
      pol.decode(box, at, i, j, k);
      double s[NVAR];
      pol.raw(true, box, at, i, j, k, s);
      if (s[URHO] == 0.) {
        report_error(err, 3, i, j, k);  // amrex::Error in the reference
      } else {
        int blo[3], bhi[3];
        pol.window(box, i, j, k, blo, bhi);
        double max_dens = s[URHO];
        int64_t pick = at;
        int pick_m = -1;
        for (int kk = -1; kk <= 1; kk++)
          for (int jj = -1; jj <= 1; jj++)
            for (int ii = -1; ii <= 1; ii++) {
              if (i + ii >= blo[0] && j + jj >= blo[1] && k + kk >= blo[2] && i + ii <= bhi[0] &&
                  j + jj <= bhi[1] && k + kk <= bhi[2]) {
                const int64_t nat = pol.idx(box, i + ii, j + jj, k + kk);
                const int mm = floor_find(key, n, (box << 40) | nat);
                // a cell reset earlier in this walk, else the pass's value
                const double r =
                    (mm >= 0 && mm < m) ? enf[int64_t(mm) * NVAR + URHO] : pol.dens(box, nat);
                if (r > max_dens) {
                  pick = nat;
                  pick_m = mm;
                  max_dens = r;
                }
              }
            }
        if (max_dens < P.small_dens) {
          double massfrac[NSPEC];
          for (int sp = 0; sp < NSPEC; ++sp) massfrac[sp] = s[UFS + sp] / s[URHO];
          const double small_e = eos_rty2e(P.gamma, P.small_temp, massfrac);
          s[URHO] = P.small_dens;
          s[UTEMP] = P.small_temp;
          s[UMX] = 0.;
          s[UMY] = 0.;
          s[UMZ] = 0.;
          s[UEINT] = P.small_dens * small_e;
          s[UEDEN] = s[UEINT];
        } else if (pick_m >= 0) {
          // a cell reset earlier (a listed cell not yet reached lies below
          // the floor, so it never is the densest at or above it)
          for (int q = 0; q < NVAR; ++q) s[q] = enf[int64_t(pick_m) * NVAR + q];
        } else {
          int pi, pj, pk;
          pol.decode(box, pick, pi, pj, pk);
          pol.raw(false, box, pick, pi, pj, pk, s);
        }
      }
      for (int q = 0; q < NVAR; ++q) enf[int64_t(m) * NVAR + q] = s[q];
    }
  }
}

// The single-level view of floor_walk: boxes of boxsz cells tile the domain.
template <int MODE>
struct LevelFloorPolicy {
  const LGeom& L;
  const KParams& P;
  const FloorArgs& a;
  __device__ void decode(int64_t, int64_t at, int& i, int& j, int& k) const {
    decode_cell(L, at, i, j, k);
  }
  __device__ void window(int64_t, int i, int j, int k, int* blo, int* bhi) const {
    const int c[3] = {i, j, k};
    for (int d = 0; d < 3; ++d) {
      const int b = (c[d] - L.dlo[d]) / L.boxsz[d];
      blo[d] = L.dlo[d] + b * L.boxsz[d];
      bhi[d] = min(blo[d] + L.boxsz[d] - 1, L.dhi[d]);
    }
  }
  __device__ int64_t idx(int64_t, int i, int j, int k) const { return L.idx(i, j, k); }
  __device__ double dens(int64_t, int64_t at) const {
    // the cleans read the array being cleaned; an update pass stored the
    // post-Saxpy state of listed cells, and for the others the stored
    // density is the post-Saxpy one too (the cleans and the gravity source
    // leave the density alone)
    if constexpr (MODE == FLOOR_CLEAN || MODE == FLOOR_EXPAND || MODE == FLOOR_INPLACE)
      return a.in[at];
    else
      return a.out[at];
  }
  __device__ void raw(bool listed, int64_t, int64_t at, int i, int j, int k, double* s) const {
    floor_raw<MODE>(L, P, a, listed, at, i, j, k, s);
  }
};

// enforce_min_density on a pass's listed cells (floor_walk), then the rest
// of the listed cells' pass: normalize_species + computeTemp (CLEAN,
// EXPAND), nothing (INPLACE: a later kernel finishes every cell), or the
// end of the step with its CFL dt (updates).  One block.  The window is the
// level box holding the cell (the reference's GPU build loops over boxes;
// its OpenMP build over tiles of them).  More than kFloorCap listed cells:
// error code 5 and the cells stay as the pass left them.  The count is
// cleared at the end, ready for the next pass.
template <int MODE>
__global__ void __launch_bounds__(1024) k_floor_fixup(LGeom L, KParams P, FloorList fl,
                                                       FloorArgs a, DevError* err) {
  extern __shared__ int64_t key[];
  const int n = *fl.count;
  if (n == 0) return;
  if (n > kFloorCap) {
    __syncthreads();
    if (threadIdx.x == 0) {
      int i, j, k;
      decode_cell(L, fl.cells[0], i, j, k);
      report_error(err, 5, i, j, k);
      *fl.count = 0;
    }
    return;
  }
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    const int64_t at = fl.cells[t];
    int i, j, k;
    decode_cell(L, at, i, j, k);
    key[t] = floor_key(L, at, i, j, k);
  }
  floor_sort(key, n);
  double* enf = fl.enforced;
  floor_walk(LevelFloorPolicy<MODE>{L, P, a}, P, key, n, enf, err);
  __syncthreads();
  for (int m = threadIdx.x; m < n; m += blockDim.x) {
    const int64_t at = key[m] & kFloorAtMask;
    int i, j, k;
    decode_cell(L, at, i, j, k);
    double s[NVAR];
    for (int q = 0; q < NVAR; ++q) s[q] = enf[int64_t(m) * NVAR + q];
    if constexpr (MODE == FLOOR_INPLACE) {
      store_cell(a.out, L, at, s);
    } else if constexpr (MODE == FLOOR_CLEAN || MODE == FLOOR_EXPAND) {
      normalize_species(s);
      compute_temp(s, P);
      if constexpr (MODE == FLOOR_CLEAN) {
        store_cell(a.out, L, at, s);
      } else {
        // the cell and every ghost cell that is its periodic image
        // (FillBoundary after normalize_species)
        int lo[3], hi[3], len[3];
        const int c[3] = {i, j, k};
        for (int d = 0; d < 3; ++d) {
          len[d] = L.dhi[d] - L.dlo[d] + 1;
          lo[d] = hi[d] = 0;
          if (L.periodic[d]) {
            while (c[d] + (lo[d] - 1) * len[d] >= L.plo[d]) --lo[d];
            while (c[d] + (hi[d] + 1) * len[d] <= L.plo[d] + L.pn[d] - 1) ++hi[d];
          }
        }
        for (int mz = lo[2]; mz <= hi[2]; ++mz)
          for (int my = lo[1]; my <= hi[1]; ++my)
            for (int mx = lo[0]; mx <= hi[0]; ++mx)
              store_cell(a.out, L, L.idx(i + mx * len[0], j + my * len[1], k + mz * len[2]), s);
      }
    } else {
      double sold[NVAR];
      for (int q = 0; q < NVAR; ++q) sold[q] = 0.0;
      if (P.add_grav_src) {
        sold[URHO] = a.S_old[at + URHO * L.sn];
        sold[UMZ] = a.S_old[at + UMZ * L.sn];
      }
      const double v = finish_step(s, sold, P, L, *a.dtp, i, j, k, err, a.post != 0);
      store_cell(a.out, L, at, s);
      if (a.bits) atomicMin(a.bits, (unsigned long long)__double_as_longlong(v));
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (fl.total) atomicAdd(fl.total, (unsigned long long)n);
    *fl.count = 0;
  }
}

// Allow the fixups of this translation unit their dynamic shared memory.
inline cudaError_t floor_prepare() {
  const void* f[] = {reinterpret_cast<const void*>(&k_floor_fixup<FLOOR_CLEAN>),
                     reinterpret_cast<const void*>(&k_floor_fixup<FLOOR_EXPAND>),
                     reinterpret_cast<const void*>(&k_floor_fixup<FLOOR_CTU>),
                     reinterpret_cast<const void*>(&k_floor_fixup<FLOOR_MOL2>),
                     reinterpret_cast<const void*>(&k_floor_fixup<FLOOR_DSDT_CTU>),
                     reinterpret_cast<const void*>(&k_floor_fixup<FLOOR_DSDT_MOL2>),
                     reinterpret_cast<const void*>(&k_floor_fixup<FLOOR_INPLACE>)};
  for (const void* k : f) {
    const cudaError_t e =
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kFloorSmem));
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

struct DtCtl {
  double cfl, max_dt, fixed_dt, initial_dt, init_shrink, change_max;
};

// estTimeStep's tail + computeInitialDt / computeNewDt for one level
// (Source/CAMR.cpp:490-635), on one thread; resets the CFL accumulator.
__global__ void k_dt_next(DtCtl c, int first, const double* fixed, unsigned long long* bits,
                          double* dt_cur, double* hist, int* nstep, int hist_cap) {
  double est;
  if (c.fixed_dt > 0.0) {
    est = c.fixed_dt;
  } else {
    double estdt = c.max_dt;
    const double max_dt_over_cfl = c.max_dt / c.cfl;
    double estdt_hydro = max_dt_over_cfl;
    const double dtc = __longlong_as_double((long long)*bits);
    estdt_hydro = dmin(estdt_hydro, dtc);
    estdt_hydro *= c.cfl;
    if (estdt_hydro < estdt) estdt = estdt_hydro;
    est = estdt;
  }
  double dt;
  if (fixed) {
    dt = *fixed;
  } else if (first) {
    double init_dt = (c.initial_dt > 0.0) ? c.initial_dt : c.init_shrink * est;
    double dt_0 = DBL_MAX;
    dt_0 = dmin(dt_0, 1 * init_dt);
    dt = dt_0 / 1;
  } else {
    double dt_min = est;
    if (c.fixed_dt <= 0.0) dt_min = dmin(dt_min, c.change_max * *dt_cur);
    double dt_0 = DBL_MAX;
    dt_0 = dmin(dt_0, 1 * dt_min);
    dt = dt_0 / 1;
  }
  *dt_cur = dt;
  const int n = *nstep;
  if (n < hist_cap) hist[n] = dt;
  *nstep = n + 1;
  *bits = (unsigned long long)__double_as_longlong(DBL_MAX);
}

__global__ void k_reset_bits(unsigned long long* bits) {
  *bits = (unsigned long long)__double_as_longlong(DBL_MAX);
}

// enforce_consistent_e (Source/CAMR.cpp:910-939) then computeTemp.
__global__ void __launch_bounds__(kBlk) k_init_finalize(LGeom L, KParams P, double* S) {
  int i, j, k;
  if (!valid_cell(L, tid(), i, j, k)) return;
  const int64_t at = L.idx(i, j, k);
  double s[NVAR];
  load_cell(S, L, at, s);
  const double rhoInv = 1.0 / s[URHO];
  const double u = s[UMX] * rhoInv;
  const double v = s[UMY] * rhoInv;
  const double w = s[UMZ] * rhoInv;
  s[UEDEN] = s[UEINT] + 0.5 * s[URHO] * (u * u + v * v + w * w);
  compute_temp(s, P);
  store_cell(S, L, at, s);
}

// Copy between a packed (NVAR, nz, ny, nx) array and the padded state.
__global__ void __launch_bounds__(kBlk) k_pack(LGeom L, const double* padded, double* packed,
                                                int to_packed) {
  int i, j, k;
  const int64_t t = tid();
  if (!valid_cell(L, t, i, j, k)) return;
  const int64_t nc = int64_t(L.dhi[0] - L.dlo[0] + 1) * (L.dhi[1] - L.dlo[1] + 1) *
                     (L.dhi[2] - L.dlo[2] + 1);
  const int64_t at = L.idx(i, j, k);
  for (int n = 0; n < NVAR; ++n) {
    if (to_packed) packed[t + n * nc] = padded[at + n * L.sn];
    else const_cast<double*>(padded)[at + n * L.sn] = packed[t + n * nc];
  }
}

}  // namespace
}  // namespace camr
