// Two-level AMR hierarchy on the device: a base level over the whole
// (periodic) domain and a fixed set of fine boxes at refinement ratio 2,
// advanced with subcycling as Amr::timeStep drives CAMR for two levels:
//
//   level 0: CAMR::CAMR_advance (Source/CAMR_advance.cpp:38-164) with the
//            flux register's CrseAdd after each hydro call
//            (Source/Hydro/CAMR_construct_hydro_source.cpp:243-248)
//   level 1: two substeps of CAMR_advance + post_timestep's clean_state, the
//            fine ghost cells filled by FillPatchTwoLevels (other fine boxes,
//            else the base level interpolated in time and space) and FineAdd
//            after each hydro call (:249-253)
//   level 0: post_timestep: reflux, avgDown, clean_state (Source/CAMR.cpp:679-718,
//            :803-851, :1048-1066)
//   dt:      computeNewDt / computeInitialDt over both levels (:566-676)
//
// Data layout: the base level is one padded domain array per state (as the
// single-level driver); each fine box owns padded arrays over its own hydro
// Space (box grown by 4, +1 face layer) carved from one pool per state.
// The fine hydro is the batched work-list plan (one launch per stage for
// all boxes); every other fine pass is one launch over all boxes' cells
// (a block prefix over the boxes, binary-searched per block).  The flux
// register keeps its sums per coarse-fine boundary cell; each boundary
// cell's contributions are summed by one thread in a fixed order, so the
// result does not depend on scheduling.  The whole coarse step is
// stream-ordered with dt and the level times in device memory, and is
// captured once into a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "level_point.cuh"

namespace camr {
namespace {

constexpr int RR = 2;  // refinement ratio

// Coarse data at a fine time: StateData::getData's choice (new, old, or
// both combined by LinComb with weights alpha, beta).
struct CoarseT {
  int mode;  // 0 new, 1 old, 2 alpha*old + beta*new
  double alpha, beta;
};

struct AmrClock {
  double tc_old, tc_new;  // level 0 old / new time
  double tf_old, tf_new;  // level 1 old / new time
  double dt0, dt1;        // dt of each level in the current coarse step
  CoarseT ct[2];          // coarse data at the fine substep's old / new time
  int nstep;
};

// The fine boxes as seen by the kernels.
struct FineDev {
  int nbox;
  const LGeom* L;          // per box: the box as the "domain" of its padded arrays
  const int64_t* off;      // per box: offset (doubles) of its arrays in each pool
  const int64_t* vb0;      // nbox+1: first block of each box's valid cells
  const int64_t* gb0;      // nbox+1: first block of each box's grown cells
  const int64_t* poff;     // per box: offset of its cells in the packed I/O array
  double* const* qf;       // nbox*3: interface p, u_n of each box's last hydro
  const int* vbox;         // per valid-cell block: its box (null: search vb0)
  const int* gbox;         // per grown-cell block: its box (null: search gb0)
};

// Coarse cell lookups (periodic wrap).
struct CoarseMap {
  const int* cmap;  // coarse valid cell -> fine box covering it, or -1
  const int* bmap;  // coarse valid cell -> flux-register boundary index, or -1
  int dlo[3], n[3];
  __device__ __forceinline__ int cell(int i, int j, int k) const {
    const int c[3] = {i, j, k};
    int w[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) w[d] = ((((c[d] - dlo[d]) % n[d]) + n[d]) % n[d]);
    return w[0] + n[0] * (w[1] + n[1] * w[2]);
  }
  // cell() of a cell inside the domain, without the periodic wrap
  __device__ __forceinline__ int cell_in(int i, int j, int k) const {
    return (i - dlo[0]) + n[0] * ((j - dlo[1]) + n[1] * (k - dlo[2]));
  }
};

__device__ __forceinline__ int floordiv2(int v) { return (v >= 0) ? v / RR : -((-v + RR - 1) / RR); }
__device__ __forceinline__ int wrapi(int v, int lo, int n) { return lo + (((v - lo) % n) + n) % n; }
// wrapi without the divisions when v is less than one period outside
// [lo, lo + n), as the coarse neighbours of a fine box's ghost shell are.
__device__ __forceinline__ int wrap_near(int v, int lo, int n) {
  int w = v - lo;
  if (w < 0) w += n;
  else if (w >= n) w -= n;
  if (unsigned(w) >= unsigned(n)) w = ((w % n) + n) % n;
  return lo + w;
}

__device__ __forceinline__ int box_of_block(const int64_t* b0, int nbox, int64_t blk) {
  int lo = 0, hi = nbox - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (b0[mid] <= blk) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ Space space_of(const LGeom& L) {
  Space sp;
  for (int d = 0; d < 3; ++d) {
    sp.lo[d] = L.plo[d];
    sp.n[d] = L.pn[d] + 1;
  }
  sp.sy = L.sy;
  sp.sz = L.sz;
  sp.sn = L.sn;
  return sp;
}

// Coarse state at time ct of component n at a (periodic) coarse cell.
__device__ __forceinline__ double coarse_at(const LGeom& Lc, const double* c_old,
                                            const double* c_new, const CoarseT& ct, int i, int j,
                                            int k, int n) {
  const int ni = Lc.dhi[0] - Lc.dlo[0] + 1, nj = Lc.dhi[1] - Lc.dlo[1] + 1,
            nk = Lc.dhi[2] - Lc.dlo[2] + 1;
  const int64_t at = Lc.idx(wrapi(i, Lc.dlo[0], ni), wrapi(j, Lc.dlo[1], nj),
                            wrapi(k, Lc.dlo[2], nk)) + n * Lc.sn;
  if (ct.mode == 0) return c_new[at];
  if (ct.mode == 1) return c_old[at];
  return ct.alpha * c_old[at] + ct.beta * c_new[at];
}

#define FINE_VALID_PROLOGUE                                          \
  const int b = F.vbox ? F.vbox[blockIdx.x] : box_of_block(F.vb0, F.nbox, blockIdx.x); \
  const LGeom& L = F.L[b];                                           \
  const int64_t t = (int64_t(blockIdx.x) - F.vb0[b]) * kBlk + threadIdx.x; \
  int i, j, k;                                                       \
  const bool ok = valid_cell(L, t, i, j, k);

// enforce_consistent_e + computeTemp on the fine valid cells
// (Source/CAMR.cpp:414-420).
__global__ void __launch_bounds__(kBlk) kf_init_finalize(FineDev F, KParams P, double* S) {
  FINE_VALID_PROLOGUE
  if (!ok) return;
  double* Sb = S + F.off[b];
  const int64_t at = L.idx(i, j, k);
  double s[NVAR];
  load_cell(Sb, L, at, s);
  const double rhoInv = 1.0 / s[URHO];
  const double u = s[UMX] * rhoInv;
  const double v = s[UMY] * rhoInv;
  const double w = s[UMZ] * rhoInv;
  s[UEDEN] = s[UEINT] + 0.5 * s[URHO] * (u * u + v * v + w * w);
  compute_temp(s, P);
  store_cell(Sb, L, at, s);
}

// S_old = clean_state(S) on the fine valid cells (the density floor's
// neighbour window is the box).
__global__ void __launch_bounds__(kBlk) kf_clean_copy(FineDev F, KParams P, const double* S,
                                                       double* out, DevError* err,
                                                       FloorList fl) {
  FINE_VALID_PROLOGUE
  if (!ok) return;
  const double* Sb = S + F.off[b];
  const int64_t at = L.idx(i, j, k);
  double s[NVAR];
  load_cell(Sb, L, at, s);
  if (s[URHO] < P.small_dens) floor_push(fl, (int64_t(b) << 40) | at);
  enforce_min_density(s, Sb, L, P, i, j, k, err);
  normalize_species(s);
  compute_temp(s, P);
  store_cell(out + F.off[b], L, at, s);
}

__global__ void __launch_bounds__(kBlk) kf_est_dt(FineDev F, KParams P, const double* S,
                                                   unsigned long long* bits) {
  FINE_VALID_PROLOGUE
  double v = DBL_MAX;
  if (ok) {
    double s[NVAR];
    load_cell(S + F.off[b], L, L.idx(i, j, k), s);
    v = cell_dt(s, L, P);
  }
  block_min_dt(v, bits);
}

// expand_state on the fine level, part 1: valid cells and the ghost cells
// that a fine box covers (through the periodic domain) take the cleaned
// value of that box's cell (enforce_min_density + normalize_species, then
// FillBoundary), then computeTemp.  The coarse-fine ghost cells are left to
// kf_interp.
__global__ void __launch_bounds__(kBlk) kf_fill(FineDev F, KParams P, CoarseMap CM,
                                                 const double* src, double* B, int3 fdlo,
                                                 int3 fdn, DevError* err, FloorList fl) {
  const int b = F.gbox ? F.gbox[blockIdx.x] : box_of_block(F.gb0, F.nbox, blockIdx.x);
  const LGeom& L = F.L[b];
  const int64_t t = (int64_t(blockIdx.x) - F.gb0[b]) * kBlk + threadIdx.x;
  int i, j, k;
  if (!padded_cell(L, t, i, j, k)) return;
  double s[NVAR];
  const bool valid = i >= L.dlo[0] && i <= L.dhi[0] && j >= L.dlo[1] && j <= L.dhi[1] &&
                     k >= L.dlo[2] && k <= L.dhi[2];
  if (valid) {
    const double* sb = src + F.off[b];
    load_cell(sb, L, L.idx(i, j, k), s);
    if (s[URHO] < P.small_dens) floor_push(fl, (int64_t(b) << 40) | L.idx(i, j, k));
    enforce_min_density(s, sb, L, P, i, j, k, err);
  } else {
    // a ghost cell lies at most NGROW cells outside its box, so within one
    // period of the fine domain; its image's coarse parent is a domain cell
    const int wi = wrap_near(i, fdlo.x, fdn.x), wj = wrap_near(j, fdlo.y, fdn.y),
              wk = wrap_near(k, fdlo.z, fdn.z);
    const int ob = CM.cmap[CM.cell_in(floordiv2(wi), floordiv2(wj), floordiv2(wk))];
    if (ob < 0) return;
    const LGeom& Lo = F.L[ob];
    const double* so = src + F.off[ob];
    load_cell(so, Lo, Lo.idx(wi, wj, wk), s);
    enforce_min_density(s, so, Lo, P, wi, wj, wk, err);
  }
  normalize_species(s);
  compute_temp(s, P);
  store_cell(B + F.off[b], L, L.idx(i, j, k), s);
}

// expand_state on the fine level, part 2: the ghost cells no fine box
// covers, one thread per coarse cell of grow(coarsened box, 2) outside the
// coarsened box and outside every fine box.  Per component the 27 coarse
// neighbours at the fine time are gathered once; the AMReX
// CellConservativeLinear slopes (ratio 2, with limiting) give the 8 fine
// children: per-direction MC-limited slopes, one factor alpha keeping the
// children inside the neighbours' min/max, child = u + ox*sx + oy*sy + oz*sz
// with o = -+1/4.  Then computeTemp on each child.
// resident 256-thread blocks per SM asked of the coarse-to-fine interpolation
// 1: the coarse-to-fine interpolation runs over a list of (coarse cell,
// component) pairs (kf_interp_list); 0: one thread per coarse cell of each
// box's grown shell walks the components (kf_interp).
// 1: the fine kernels read their block's box from a per-block table; 0:
// each block binary-searches the boxes' first blocks.
#ifndef CAMR_FINE_BLOCKMAP
#define CAMR_FINE_BLOCKMAP 1
#endif
#ifndef CAMR_INTERP_LIST
#define CAMR_INTERP_LIST 1
#endif
#ifndef CAMR_MINB_INTERP
#define CAMR_MINB_INTERP 3
#endif
__global__ void __launch_bounds__(kBlk, CAMR_MINB_INTERP) kf_interp(FineDev F, KParams P, CoarseMap CM,
                                                   LGeom Lc, const double* c_old,
                                                   const double* c_new, const CoarseT* ctp,
                                                   const int64_t* ib0, double* B) {
  const int b = box_of_block(ib0, F.nbox, blockIdx.x);
  const LGeom& L = F.L[b];
  const int64_t t = (int64_t(blockIdx.x) - ib0[b]) * kBlk + threadIdx.x;
  int clo[3], cn[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    clo[d] = floordiv2(L.dlo[d]) - 2;
    cn[d] = floordiv2(L.dhi[d]) - floordiv2(L.dlo[d]) + 1 + 4;
  }
  if (t >= int64_t(cn[0]) * cn[1] * cn[2]) return;
  const int64_t nxy = int64_t(cn[0]) * cn[1];
  const int kk = int(t / nxy);
  const int64_t r = t - int64_t(kk) * nxy;
  const int jj = int(r / cn[0]);
  const int ii = int(r - int64_t(jj) * cn[0]);
  if (ii >= 2 && ii < cn[0] - 2 && jj >= 2 && jj < cn[1] - 2 && kk >= 2 && kk < cn[2] - 2) return;
  const int ci = clo[0] + ii, cj = clo[1] + jj, ck = clo[2] + kk;
  if (CM.cmap[CM.cell(ci, cj, ck)] >= 0) return;
  const CoarseT ct = *ctp;
  double* Bb = B + F.off[b];
  const int64_t at0 = L.idx(RR * ci, RR * cj, RR * ck);
  const int64_t cstep[3] = {1, L.sy, L.sz};
  for (int n = 0; n < NVAR; ++n) {
    double v[27];
#pragma unroll
    for (int dk = -1; dk <= 1; ++dk)
#pragma unroll
      for (int dj = -1; dj <= 1; ++dj)
#pragma unroll
        for (int di = -1; di <= 1; ++di)
          v[(dk + 1) * 9 + (dj + 1) * 3 + (di + 1)] =
              coarse_at(Lc, c_old, c_new, ct, ci + di, cj + dj, ck + dk, n);
    const double uc = v[13];
    const double up[3] = {v[14], v[16], v[22]};
    const double um[3] = {v[12], v[10], v[4]};
    double sl[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double dc = 0.5 * (up[d] - um[d]);
      const double df = 2.0 * (up[d] - uc);
      const double db = 2.0 * (uc - um[d]);
      double sv = (df * db >= 0.0) ? dmin(fabs(df), fabs(db)) : 0.0;
      sv = copysign(1.0, dc) * dmin(sv, fabs(dc));
      sl[d] = sv;
    }
    double alpha = 1.0;
    if (sl[0] != 0.0 || sl[1] != 0.0 || sl[2] != 0.0) {
      const double dumax = fabs(sl[0]) * 0.25 + fabs(sl[1]) * 0.25 + fabs(sl[2]) * 0.25;
      double umax = uc, umin = uc;
#pragma unroll
      for (int q = 0; q < 27; ++q) {
        umax = dmax(umax, v[q]);
        umin = dmin(umin, v[q]);
      }
      if (dumax * alpha > (umax - uc)) alpha = (umax - uc) / dumax;
      if (dumax * alpha > (uc - umin)) alpha = (uc - umin) / dumax;
    }
    const double sa[3] = {sl[0] * alpha, sl[1] * alpha, sl[2] * alpha};
    double* Bn = Bb + at0 + int64_t(n) * L.sn;
#pragma unroll
    for (int kc = 0; kc < RR; ++kc)
#pragma unroll
      for (int jc = 0; jc < RR; ++jc)
#pragma unroll
        for (int ic = 0; ic < RR; ++ic) {
          const double ox = ic ? 0.25 : -0.25, oy = jc ? 0.25 : -0.25, oz = kc ? 0.25 : -0.25;
          Bn[ic * cstep[0] + jc * cstep[1] + kc * cstep[2]] =
              uc + ox * sa[0] + oy * sa[1] + oz * sa[2];
        }
  }
#pragma unroll 1
  for (int q = 0; q < 8; ++q) {
    const int64_t at = at0 + (q & 1) * cstep[0] + ((q >> 1) & 1) * cstep[1] + (q >> 2) * cstep[2];
    double s[NVAR];
    load_cell(Bb, L, at, s);
    compute_temp(s, P);
    store_cell(Bb, L, at, s);
  }
}

// The same interpolation spread over (coarse cell, component) pairs: the
// coarse ghost cells to fill are listed once when the hierarchy is built
// (box, coarse i, j, k, in kf_interp's order), a block takes kInterpItems
// of them and one thread per (cell, component) gathers that component's 27
// neighbours and writes its 8 children; after a barrier one thread per
// child runs computeTemp.  Each value is computed by the arithmetic of
// kf_interp, so the two give the same bits; this form has ten independent
// gathers per cell in flight instead of one component after another.
constexpr int kInterpItems = kBlk / NVAR;
static_assert(kInterpItems * RR * RR * RR <= kBlk, "one thread per child");
__global__ void __launch_bounds__(kBlk) kf_interp_list(FineDev F, KParams P, LGeom Lc,
                                                        const double* c_old, const double* c_new,
                                                        const CoarseT* ctp, const int4* items,
                                                        int64_t nitems, double* B) {
  const int slot = int(threadIdx.x) % kInterpItems;
  const int n = int(threadIdx.x) / kInterpItems;
  const int64_t first = int64_t(blockIdx.x) * kInterpItems;
  const int64_t it = first + slot;
  if (n < NVAR && it < nitems) {
    const int4 c = items[it];
    const int b = c.x, ci = c.y, cj = c.z, ck = c.w;
    const LGeom& L = F.L[b];
    const CoarseT ct = *ctp;
    // the neighbours' periodic images (the indices coarse_at reads)
    int w[3][3];
    const int cc[3] = {ci, cj, ck};
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
      for (int o = 0; o < 3; ++o) w[d][o] = wrap_near(cc[d] + o - 1, Lc.dlo[d], Lc.dhi[d] - Lc.dlo[d] + 1);
    double v[27];
#pragma unroll
    for (int dk = 0; dk < 3; ++dk)
#pragma unroll
      for (int dj = 0; dj < 3; ++dj)
#pragma unroll
        for (int di = 0; di < 3; ++di) {
          const int64_t at = Lc.idx(w[0][di], w[1][dj], w[2][dk]) + n * Lc.sn;
          double x;
          if (ct.mode == 0) x = c_new[at];
          else if (ct.mode == 1) x = c_old[at];
          else x = ct.alpha * c_old[at] + ct.beta * c_new[at];
          v[dk * 9 + dj * 3 + di] = x;
        }
    const double uc = v[13];
    const double up[3] = {v[14], v[16], v[22]};
    const double um[3] = {v[12], v[10], v[4]};
    double sl[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double dc = 0.5 * (up[d] - um[d]);
      const double df = 2.0 * (up[d] - uc);
      const double db = 2.0 * (uc - um[d]);
      double sv = (df * db >= 0.0) ? dmin(fabs(df), fabs(db)) : 0.0;
      sv = copysign(1.0, dc) * dmin(sv, fabs(dc));
      sl[d] = sv;
    }
    double alpha = 1.0;
    if (sl[0] != 0.0 || sl[1] != 0.0 || sl[2] != 0.0) {
      const double dumax = fabs(sl[0]) * 0.25 + fabs(sl[1]) * 0.25 + fabs(sl[2]) * 0.25;
      double umax = uc, umin = uc;
#pragma unroll
      for (int q = 0; q < 27; ++q) {
        umax = dmax(umax, v[q]);
        umin = dmin(umin, v[q]);
      }
      if (dumax * alpha > (umax - uc)) alpha = (umax - uc) / dumax;
      if (dumax * alpha > (uc - umin)) alpha = (uc - umin) / dumax;
    }
    const double sa[3] = {sl[0] * alpha, sl[1] * alpha, sl[2] * alpha};
    double* Bn = B + F.off[b] + L.idx(RR * ci, RR * cj, RR * ck) + int64_t(n) * L.sn;
#pragma unroll
    for (int kc = 0; kc < RR; ++kc)
#pragma unroll
      for (int jc = 0; jc < RR; ++jc)
#pragma unroll
        for (int ic = 0; ic < RR; ++ic) {
          const double ox = ic ? 0.25 : -0.25, oy = jc ? 0.25 : -0.25, oz = kc ? 0.25 : -0.25;
          Bn[ic + jc * L.sy + kc * L.sz] = uc + ox * sa[0] + oy * sa[1] + oz * sa[2];
        }
  }
  __syncthreads();
  // computeTemp on the children, one thread each
  const int q = int(threadIdx.x) % (RR * RR * RR);
  const int64_t cit = first + int(threadIdx.x) / (RR * RR * RR);
  if (int(threadIdx.x) < kInterpItems * RR * RR * RR && cit < nitems) {
    const int4 c = items[cit];
    const LGeom& L = F.L[c.x];
    double* Bb = B + F.off[c.x];
    const int64_t at = L.idx(RR * c.y + (q & 1), RR * c.z + ((q >> 1) & 1), RR * c.w + (q >> 2));
    double s[NVAR];
    load_cell(Bb, L, at, s);
    compute_temp(s, P);
    store_cell(Bb, L, at, s);
  }
}

struct FinePools {
  double* flx[3];
};

__device__ __forceinline__ FluxPtrs fine_fluxes(const FineDev& F, const FinePools& fp, int b) {
  FluxPtrs r;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    r.f[d] = fp.flx[d] + F.off[b];
    r.q[d] = F.qf[3 * b + d];
  }
  return r;
}

// The fine updates' post-Saxpy states of cell (i,j,k) of box b (the fixup
// recomputes them for neighbours of cells below the density floor).  CTU:
// S = Sborder (+ dt*src_old) + dt*dSdt; sold holds the old density and z
// momentum the gravity terms read (zero otherwise).
__device__ __forceinline__ void fine_ctu_raw(const FineDev& F, const FinePools& fpool,
                                             const KParams& P, double dt, const double* B,
                                             const double* S_old, int b, const LGeom& L, int i,
                                             int j, int k, double* s, double* sold) {
  const int64_t at = L.idx(i, j, k);
  const int64_t o = F.off[b];
  double hs[NVAR];
  load_cell(B + o, L, at, s);
#pragma unroll
  for (int n = 0; n < NVAR; ++n) sold[n] = 0.0;
  if (P.add_grav_src) {
    sold[URHO] = S_old[o + at + URHO * L.sn];
    sold[UMZ] = S_old[o + at + UMZ * L.sn];
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
  const FluxPtrs fp = fine_fluxes(F, fpool, b);
  cell_dsdt(L, space_of(L), i, j, k, fp.f, fp.q, hs);
#pragma unroll
  for (int n = 0; n < NVAR; ++n) s[n] += dt * hs[n];
}

// MOL stage 2: S = 0.5*Sborder2 + 0.5*S_old + 0.5*dt*k2; sold = S_old.
__device__ __forceinline__ void fine_mol2_raw(const FineDev& F, const FinePools& fpool,
                                              double dt, const double* B2, const double* S_old,
                                              int b, const LGeom& L, int i, int j, int k,
                                              double* s, double* sold) {
  const int64_t at = L.idx(i, j, k);
  const int64_t o = F.off[b];
  double bb[NVAR], hs[NVAR];
  load_cell(B2 + o, L, at, bb);
  load_cell(S_old + o, L, at, sold);
#pragma unroll
  for (int n = 0; n < NVAR; ++n) s[n] = 0.5 * bb[n] + 0.5 * sold[n];
  const FluxPtrs fp = fine_fluxes(F, fpool, b);
  cell_dsdt(L, space_of(L), i, j, k, fp.f, fp.q, hs);
#pragma unroll
  for (int n = 0; n < NVAR; ++n) s[n] += 0.5 * dt * hs[n];
}

// Fine-level density-floor list entry: box << 40 | index in the box's arrays.
__device__ __forceinline__ void fine_floor_push(const FloorList& fl, int b, int64_t at) {
  floor_push(fl, (int64_t(b) << 40) | at);
}

// CTU fine update, then the step's clean_states and post_timestep's (the
// finest level cleans its own).  A cell below the density floor keeps its
// post-Saxpy state and joins the list (kf_floor_fixup finishes it).
__global__ void __launch_bounds__(kBlk, CAMR_MINB_UPDATE) kf_update_ctu(FineDev F, FinePools fpool, KParams P,
                                                       const double* dtp, const double* B,
                                                       const double* S_old, double* S,
                                                       unsigned long long* bits, DevError* err,
                                                       FloorList fl) {
  FINE_VALID_PROLOGUE
  double v = DBL_MAX;
  if (ok) {
    const double dt = *dtp;
    const int64_t at = L.idx(i, j, k);
    double s[NVAR], sold[NVAR];
    fine_ctu_raw(F, fpool, P, dt, B, S_old, b, L, i, j, k, s, sold);
    if (s[URHO] < P.small_dens) fine_floor_push(fl, b, at);
    else v = finish_step(s, sold, P, L, dt, i, j, k, err, true);
    store_cell(S + F.off[b], L, at, s);
  }
  if (bits) block_min_dt(v, bits);
}

__global__ void __launch_bounds__(kBlk) kf_update_mol1(FineDev F, FinePools fpool, KParams P,
                                                        const double* dtp, const double* B,
                                                        const double* S_old, double* S) {
  FINE_VALID_PROLOGUE
  if (!ok) return;
  const double dt = *dtp;
  const int64_t at = L.idx(i, j, k);
  const int64_t o = F.off[b];
  double s[NVAR], hs[NVAR];
  load_cell(B + o, L, at, s);
  if (P.add_grav_src) {
    double src[NVAR];
#pragma unroll
    for (int n = 0; n < NVAR; ++n) src[n] = 0.0;
    src[UMZ] = P.const_grav * S_old[o + at + URHO * L.sn];
    src[UEDEN] = P.const_grav * S_old[o + at + UMZ * L.sn];
#pragma unroll
    for (int n = 0; n < NVAR; ++n) s[n] += dt * src[n];
  }
  const FluxPtrs fp = fine_fluxes(F, fpool, b);
  cell_dsdt(L, space_of(L), i, j, k, fp.f, fp.q, hs);
#pragma unroll
  for (int n = 0; n < NVAR; ++n) s[n] += dt * hs[n];
  store_cell(S + o, L, at, s);
}

__global__ void __launch_bounds__(kBlk, CAMR_MINB_UPDATE) kf_update_mol2(FineDev F, FinePools fpool, KParams P,
                                                        const double* dtp, const double* B2,
                                                        const double* S_old, double* S,
                                                        unsigned long long* bits, DevError* err,
                                                        FloorList fl) {
  FINE_VALID_PROLOGUE
  double v = DBL_MAX;
  if (ok) {
    const double dt = *dtp;
    const int64_t at = L.idx(i, j, k);
    double s[NVAR], sold[NVAR];
    fine_mol2_raw(F, fpool, dt, B2, S_old, b, L, i, j, k, s, sold);
    if (s[URHO] < P.small_dens) fine_floor_push(fl, b, at);
    else v = finish_step(s, sold, P, L, dt, i, j, k, err, true);
    store_cell(S + F.off[b], L, at, s);
  }
  if (bits) block_min_dt(v, bits);
}

// The passes of the fine level whose cells below the density floor
// kf_floor_fixup finishes.
enum { FFLOOR_CLEAN = 0, FFLOOR_FILL = 1, FFLOOR_CTU = 2, FFLOOR_MOL2 = 3 };

struct FineFloorArgs {
  const double* in;      // CLEAN / FILL: the pool being cleaned
  double* out;           // CLEAN: S_old; FILL: Sborder; CTU / MOL2: S
  const double* B;       // CTU / MOL2: the stage's Sborder
  const double* S_old;
  FinePools fp;
  const double* dtp;
  unsigned long long* bits;  // CFL minimum of the updates (may be null)
  int3 fdlo, fdn;        // the fine domain (FILL: periodic images)
};

// The fine level's view of floor_walk: each fine box is its own window.
template <int MODE>
struct FineFloorPolicy {
  const FineDev& F;
  const KParams& P;
  const FineFloorArgs& a;
  __device__ void decode(int64_t box, int64_t at, int& i, int& j, int& k) const {
    decode_cell(F.L[box], at, i, j, k);
  }
  __device__ void window(int64_t box, int, int, int, int* blo, int* bhi) const {
    const LGeom& L = F.L[box];
    for (int d = 0; d < 3; ++d) {
      blo[d] = L.dlo[d];
      bhi[d] = L.dhi[d];
    }
  }
  __device__ int64_t idx(int64_t box, int i, int j, int k) const { return F.L[box].idx(i, j, k); }
  __device__ double dens(int64_t box, int64_t at) const {
    // as in the single-level fixup: the updates' stored densities are the
    // post-Saxpy ones for every cell
    if constexpr (MODE == FFLOOR_CLEAN || MODE == FFLOOR_FILL) return a.in[F.off[box] + at];
    else return a.out[F.off[box] + at];
  }
  __device__ void raw(bool listed, int64_t box, int64_t at, int i, int j, int k,
                      double* s) const {
    const LGeom& L = F.L[box];
    const int b = int(box);
    if constexpr (MODE == FFLOOR_CLEAN || MODE == FFLOOR_FILL) {
      load_cell(a.in + F.off[b], L, at, s);
    } else if (listed) {
      load_cell(a.out + F.off[b], L, at, s);
    } else {
      double sold[NVAR];
      if constexpr (MODE == FFLOOR_CTU)
        fine_ctu_raw(F, a.fp, P, *a.dtp, a.B, a.S_old, b, L, i, j, k, s, sold);
      else
        fine_mol2_raw(F, a.fp, *a.dtp, a.B, a.S_old, b, L, i, j, k, s, sold);
    }
  }
};

// enforce_min_density on the fine cells a pass listed (floor_walk, each box
// its own window as in the reference's MFIter loop), then the rest of the
// pass for them: CLEAN normalize_species + computeTemp; FILL the same, into
// the cell and into every ghost cell of any fine box that is its image
// (FillBoundary); CTU / MOL2 the end of the step and its CFL dt.  One
// block; more than kFloorCap cells: error code 5.
template <int MODE>
__global__ void __launch_bounds__(1024) kf_floor_fixup(FineDev F, KParams P, FloorList fl,
                                                        FineFloorArgs a, DevError* err) {
  extern __shared__ int64_t key[];
  const int n = *fl.count;
  if (n == 0) return;
  if (n > kFloorCap) {
    __syncthreads();
    if (threadIdx.x == 0) {
      const int64_t c = fl.cells[0];
      int i, j, k;
      decode_cell(F.L[c >> 40], c & kFloorAtMask, i, j, k);
      report_error(err, 5, i, j, k);
      *fl.count = 0;
    }
    return;
  }
  for (int t = threadIdx.x; t < n; t += blockDim.x) key[t] = fl.cells[t];
  floor_sort(key, n);
  double* enf = fl.enforced;
  floor_walk(FineFloorPolicy<MODE>{F, P, a}, P, key, n, enf, err);
  __syncthreads();
  for (int m = threadIdx.x; m < n; m += blockDim.x) {
    const int b = int(key[m] >> 40);
    const int64_t at = key[m] & kFloorAtMask;
    const LGeom& L = F.L[b];
    int i, j, k;
    decode_cell(L, at, i, j, k);
    double s[NVAR];
    for (int q = 0; q < NVAR; ++q) s[q] = enf[int64_t(m) * NVAR + q];
    if constexpr (MODE == FFLOOR_CLEAN || MODE == FFLOOR_FILL) {
      normalize_species(s);
      compute_temp(s, P);
      store_cell(a.out + F.off[b], L, at, s);
      if constexpr (MODE == FFLOOR_FILL) {
        const int len[3] = {a.fdn.x, a.fdn.y, a.fdn.z};
        const int c[3] = {i, j, k};
        for (int ob = 0; ob < F.nbox; ++ob) {
          const LGeom& Lo = F.L[ob];
          for (int mz = -1; mz <= 1; ++mz)
            for (int my = -1; my <= 1; ++my)
              for (int mx = -1; mx <= 1; ++mx) {
                const int m3[3] = {mx, my, mz};
                int g[3];
                bool in_pad = true, in_valid = true;
                for (int d = 0; d < 3; ++d) {
                  g[d] = c[d] + m3[d] * len[d];
                  in_pad = in_pad && g[d] >= Lo.plo[d] && g[d] <= Lo.plo[d] + Lo.pn[d] - 1;
                  in_valid = in_valid && g[d] >= Lo.dlo[d] && g[d] <= Lo.dhi[d];
                }
                if (in_pad && !in_valid)
                  store_cell(a.out + F.off[ob], Lo, Lo.idx(g[0], g[1], g[2]), s);
              }
        }
      }
    } else {
      double sold[NVAR];
      for (int q = 0; q < NVAR; ++q) sold[q] = 0.0;
      if (P.add_grav_src) {
        sold[URHO] = a.S_old[F.off[b] + at + URHO * L.sn];
        sold[UMZ] = a.S_old[F.off[b] + at + UMZ * L.sn];
      }
      const double v = finish_step(s, sold, P, L, *a.dtp, i, j, k, err, true);
      store_cell(a.out + F.off[b], L, at, s);
      if (a.bits) atomicMin(a.bits, (unsigned long long)__double_as_longlong(v));
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (fl.total) atomicAdd(fl.total, (unsigned long long)n);
    *fl.count = 0;
  }
}

// Allow the fine fixups their dynamic shared memory (and this translation
// unit's single-level ones).
cudaError_t kf_floor_prepare() {
  const void* f[] = {reinterpret_cast<const void*>(&kf_floor_fixup<FFLOOR_CLEAN>),
                     reinterpret_cast<const void*>(&kf_floor_fixup<FFLOOR_FILL>),
                     reinterpret_cast<const void*>(&kf_floor_fixup<FFLOOR_CTU>),
                     reinterpret_cast<const void*>(&kf_floor_fixup<FFLOOR_MOL2>)};
  for (const void* k : f) {
    const cudaError_t e =
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kFloorSmem));
    if (e != cudaSuccess) return e;
  }
  return floor_prepare();
}

// Packed (per box (NVAR, nz, ny, nx), boxes back to back) <-> fine pools.
__global__ void __launch_bounds__(kBlk) kf_pack(FineDev F, double* pool, double* packed,
                                                 int to_packed) {
  FINE_VALID_PROLOGUE
  if (!ok) return;
  const int64_t nc = int64_t(L.dhi[0] - L.dlo[0] + 1) * (L.dhi[1] - L.dlo[1] + 1) *
                     (L.dhi[2] - L.dlo[2] + 1);
  const int64_t at = F.off[b] + L.idx(i, j, k);
  double* pk = packed + F.poff[b];
  for (int n = 0; n < NVAR; ++n) {
    if (to_packed) pk[t + n * nc] = pool[at + n * L.sn];
    else pool[at + n * L.sn] = pk[t + n * nc];
  }
}

// Flux register, coarse side (YAFluxRegister::CrseAdd): per boundary cell,
// remove the coarse flux through each face shared with a fine-covered cell
// (x-, x+, y-, y+, z-, z+), scaled by fac*dt/vol (area-weighted fluxes).
struct FluxRegDev {
  int nbnd;
  const int* cell;     // nbnd*3 coarse i, j, k
  const int* mask;     // nbnd: bit 2d = low neighbour in d is fine, bit 2d+1 = high
  const int* cstart;   // nbnd+1: range of each cell's fine contributions
  const int4* contrib; // (box, dir, side, 0), in FineAdd's order
  double* d;           // NVAR*nbnd, component-major: CrseAdd sums
  double* cfp;         // NVAR*nbnd: FineAdd sums
};

__global__ void __launch_bounds__(kBlk) k_crse_add(FluxRegDev R, LGeom Lc, const double* f0,
                                                    const double* f1, const double* f2,
                                                    const double* dtp, double fac, double vol) {
  const int64_t c = tid();
  if (c >= R.nbnd) return;
  const double dtdx = (fac * *dtp) / vol;
  const int i = R.cell[3 * c], j = R.cell[3 * c + 1], k = R.cell[3 * c + 2];
  const int m = R.mask[c];
  const double* f[3] = {f0, f1, f2};
  const int64_t at = Lc.idx(i, j, k);
  const int64_t step[3] = {1, Lc.sy, Lc.sz};
  for (int n = 0; n < NVAR; ++n) {
    double d = R.d[c + int64_t(n) * R.nbnd];
#pragma unroll
    for (int dd = 0; dd < 3; ++dd) {
      if (m & (1 << (2 * dd))) d -= dtdx * f[dd][at + n * Lc.sn];
      if (m & (1 << (2 * dd + 1))) d += dtdx * f[dd][at + step[dd] + n * Lc.sn];
    }
    R.d[c + int64_t(n) * R.nbnd] = d;
  }
}

// Flux register, fine side (YAFluxRegister::FineAdd): each boundary cell
// adds, in box order, the fluxes of the 4 fine faces of each fine box side
// it touches (slower transverse index outer), scaled by
// fac*dt_f/(vol_f*ratio^3); subtracted on a box's low side, added on its
// high side.
__global__ void __launch_bounds__(kBlk) k_fine_add(FluxRegDev R, FineDev F, FinePools fpool,
                                                    const double* dtp, double fac, double volf8) {
  const int64_t c = tid();
  if (c >= R.nbnd) return;
  const double dtdx = (fac * *dtp) / volf8;
  const int cc[3] = {R.cell[3 * c], R.cell[3 * c + 1], R.cell[3 * c + 2]};
  const int q0 = R.cstart[c], q1 = R.cstart[c + 1];
  for (int n = 0; n < NVAR; ++n) {
    double acc = R.cfp[c + int64_t(n) * R.nbnd];
    for (int q = q0; q < q1; ++q) {
      const int4 ct = R.contrib[q];
      const int b = ct.x, d = ct.y, side = ct.z;
      const LGeom& L = F.L[b];
      const int t1 = (d == 0) ? 1 : 0;
      const int t2 = (d == 2) ? 1 : 2;
      const int fface = side ? L.dhi[d] + 1 : L.dlo[d];
      const double* fl = fpool.flx[d] + F.off[b] + int64_t(n) * L.sn;
      for (int a2 = 0; a2 < RR; ++a2)
        for (int a1 = 0; a1 < RR; ++a1) {
          int fi[3];
          fi[d] = fface;
          fi[t1] = RR * cc[t1] + a1;
          fi[t2] = RR * cc[t2] + a2;
          const double v = dtdx * fl[L.idx(fi[0], fi[1], fi[2])];
          if (side) acc += v;
          else acc -= v;
        }
    }
    R.cfp[c + int64_t(n) * R.nbnd] = acc;
  }
}

// Average of the 8 fine cells over coarse cell (i,j,k), component n
// (amrex_avgdown: kr, jr, ir order, then times 1/8).
__device__ __forceinline__ double avg_down_cell(const FineDev& F, const double* S1, int b, int i,
                                                int j, int k, int n) {
  const LGeom& L = F.L[b];
  const double* sb = S1 + F.off[b] + int64_t(n) * L.sn;
  double c = 0.0;
  for (int kr = 0; kr < RR; ++kr)
    for (int jr = 0; jr < RR; ++jr)
      for (int ir = 0; ir < RR; ++ir) c += sb[L.idx(RR * i + ir, RR * j + jr, RR * k + kr)];
  const double volfrac = 1.0 / static_cast<double>(RR * RR * RR);
  return volfrac * c;
}

// post_timestep on level 0 (Source/CAMR.cpp:679-718), part 1: reflux (the
// flux-register sums) and avgDown (covered cells replaced by the average of
// the fine cells), left raw in S0; cells below the density floor join the
// list (k_floor_fixup<FLOOR_INPLACE> resets them in the reference's order).
__global__ void __launch_bounds__(kBlk) k_coarse_raw(LGeom Lc, KParams P, CoarseMap CM,
                                                      FluxRegDev R, FineDev F,
                                                      const double* S1, double* S0,
                                                      FloorList fl) {
  int i, j, k;
  if (!valid_cell(Lc, tid(), i, j, k)) return;
  const int64_t at = Lc.idx(i, j, k);
  const int c = CM.cell_in(i, j, k);
  const int bi = CM.bmap[c];
  const int ob = CM.cmap[c];
  double s[NVAR];
  load_cell(S0, Lc, at, s);
#pragma unroll
  for (int n = 0; n < NVAR; ++n) {
    const double corr =
        (bi >= 0) ? R.d[bi + int64_t(n) * R.nbnd] + R.cfp[bi + int64_t(n) * R.nbnd] : 0.0 + 0.0;
    s[n] = s[n] + corr;
  }
  if (ob >= 0) {
    for (int n = 0; n < NVAR; ++n) s[n] = avg_down_cell(F, S1, ob, i, j, k, n);
  }
  if (s[URHO] < P.small_dens) floor_push(fl, at);
  store_cell(S0, Lc, at, s);
}

// Part 2: the rest of clean_state (normalize_species, computeTemp) on every
// cell and the cell's CFL dt for the next step.
__global__ void __launch_bounds__(kBlk) k_coarse_finish(LGeom Lc, KParams P, double* S0,
                                                         unsigned long long* bits,
                                                         DevError* err) {
  int i, j, k;
  double v = DBL_MAX;
  if (valid_cell(Lc, tid(), i, j, k)) {
    const int64_t at = Lc.idx(i, j, k);
    double s[NVAR];
    load_cell(S0, Lc, at, s);
    if (!(s[URHO] >= P.small_dens)) report_error(err, floor_code(s[URHO], P), i, j, k);
    normalize_species(s);
    compute_temp(s, P);
    store_cell(S0, Lc, at, s);
    v = cell_dt(s, Lc, P);
  }
  block_min_dt(v, bits);
}

// post_init's avgDown (no clean).
__global__ void __launch_bounds__(kBlk) k_init_avgdown(LGeom Lc, CoarseMap CM, FineDev F,
                                                        const double* S1, double* S0) {
  int i, j, k;
  if (!valid_cell(Lc, tid(), i, j, k)) return;
  const int ob = CM.cmap[CM.cell_in(i, j, k)];
  if (ob < 0) return;
  const int64_t at = Lc.idx(i, j, k);
  for (int n = 0; n < NVAR; ++n) S0[at + n * Lc.sn] = avg_down_cell(F, S1, ob, i, j, k, n);
}

__device__ __forceinline__ double est_tail(const DtCtl& c, unsigned long long bits) {
  if (c.fixed_dt > 0.0) return c.fixed_dt;
  double estdt = c.max_dt;
  const double max_dt_over_cfl = c.max_dt / c.cfl;
  double estdt_hydro = max_dt_over_cfl;
  const double dtc = __longlong_as_double((long long)bits);
  estdt_hydro = dmin(estdt_hydro, dtc);
  estdt_hydro *= c.cfl;
  if (estdt_hydro < estdt) estdt = estdt_hydro;
  return estdt;
}

// computeInitialDt / computeNewDt over both levels (n_cycle = 1, 2), the
// level-0 time update (swapTimeLevels), and the CFL accumulators' reset.
__global__ void k_amr_dt(DtCtl c, int first, unsigned long long* bits0,
                         unsigned long long* bits1, AmrClock* ck, double* hist, int hist_cap) {
  double dtm[2] = {est_tail(c, *bits0), est_tail(c, *bits1)};
  const double dtl[2] = {ck->dt0, ck->dt1};
  for (int l = 0; l < 2; ++l) {
    if (first) dtm[l] = (c.initial_dt > 0.0) ? c.initial_dt : c.init_shrink * dtm[l];
    else if (c.fixed_dt <= 0.0) dtm[l] = dmin(dtm[l], c.change_max * dtl[l]);
  }
  double dt_0 = DBL_MAX;
  int nf = 1;
  for (int l = 0; l < 2; ++l) {
    nf *= (l == 0) ? 1 : RR;
    dt_0 = dmin(dt_0, nf * dtm[l]);
  }
  ck->dt0 = dt_0 / 1;
  ck->dt1 = dt_0 / RR;
  ck->tc_old = ck->tc_new;
  ck->tc_new = ck->tc_new + ck->dt0;
  const int n = ck->nstep;
  if (n < hist_cap) {
    hist[2 * n] = ck->dt0;
    hist[2 * n + 1] = ck->dt1;
  }
  ck->nstep = n + 1;
  *bits0 = (unsigned long long)__double_as_longlong(DBL_MAX);
  *bits1 = (unsigned long long)__double_as_longlong(DBL_MAX);
}

__device__ __forceinline__ CoarseT coarse_time(double t0, double t1, double t) {
  CoarseT r;
  r.alpha = 0.0;
  r.beta = 0.0;
  const double teps = (t1 - t0) * 1.e-3;
  if (t > t1 - teps && t < t1 + teps) {
    r.mode = 0;
  } else if (t > t0 - teps && t < t0 + teps) {
    r.mode = 1;
  } else {
    r.mode = 2;
    r.alpha = (t1 - t) / (t1 - t0);
    r.beta = (t - t0) / (t1 - t0);
  }
  return r;
}

// Fine substep's swapTimeLevels and the coarse data choice at its old and
// new times (StateData::getData with teps = 1e-3 (t1 - t0)).
__global__ void k_fine_clock(AmrClock* ck) {
  ck->tf_old = ck->tf_new;
  ck->tf_new = ck->tf_new + ck->dt1;
  ck->ct[0] = coarse_time(ck->tc_old, ck->tc_new, ck->tf_old);
  ck->ct[1] = coarse_time(ck->tc_old, ck->tc_new, ck->tf_new);
}

__global__ void k_reset_bits2(unsigned long long* a, unsigned long long* b) {
  *a = (unsigned long long)__double_as_longlong(DBL_MAX);
  *b = (unsigned long long)__double_as_longlong(DBL_MAX);
}

template <class T>
cudaError_t upload(T** dst, const std::vector<T>& v, cudaStream_t st) {
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(dst), sizeof(T) * std::max<size_t>(1, v.size()));
  if (e == cudaSuccess && !v.empty())
    e = cudaMemcpyAsync(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, st);
  return e;
}

}  // namespace
}  // namespace camr

using namespace camr;

struct camr_amr {
  camr_hydro_params hp;
  KParams P;
  camr_level_desc desc;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  // level 0
  LGeom Lc;
  int64_t ncell0 = 0;
  double *S0 = nullptr, *S0_old = nullptr, *B0 = nullptr, *B0_2 = nullptr;
  double* flx0[3] = {nullptr, nullptr, nullptr};
  double* work0 = nullptr;
  Work w0;
  // level 1
  int nbox = 0;
  int64_t ncell1 = 0;
  int64_t pool = 0;  // doubles per state pool
  double *S1 = nullptr, *S1_old = nullptr, *B1 = nullptr;
  double* flx1[3] = {nullptr, nullptr, nullptr};
  std::vector<int64_t> h_vb0, h_gb0, h_ib0;
  LGeom* d_L = nullptr;
  int64_t *d_off = nullptr, *d_vb0 = nullptr, *d_gb0 = nullptr, *d_poff = nullptr,
          *d_ib0 = nullptr;
  int4* d_icell = nullptr;  // coarse ghost cells that kf_interp_list fills
  int64_t n_icell = 0;
  int *d_vbox = nullptr, *d_gbox = nullptr;  // box of each valid / grown block
  double** d_qf = nullptr;
  camr_batch* plan = nullptr;
  int fdlo[3], fdn[3];
  // flux register and coarse maps
  int nbnd = 0;
  int *d_cmap = nullptr, *d_bmap = nullptr, *d_bcell = nullptr, *d_mask = nullptr,
      *d_cstart = nullptr;
  int4* d_contrib = nullptr;
  double *d_reg = nullptr, *d_cfp = nullptr;
  // control
  AmrClock* clock = nullptr;
  double* hist = nullptr;
  int hist_cap = 1 << 14;
  unsigned long long *bits0 = nullptr, *bits1 = nullptr;
  DevError* err = nullptr;
  FloorList floor;  // cells below the density floor of the current pass (both levels)
  double *staging0 = nullptr, *staging1 = nullptr;
  int fine_mode = CAMR_BATCH_PERSISTENT;
  int steps_taken = 0;
  bool restart_est = false;  // next step: CFL estimate of the restored state, then computeNewDt
  bool graph_ready = false;
  cudaGraphExec_t graph;
  int64_t kernels_per_step = 0;

  FineDev fine() const {
    FineDev F;
    F.nbox = nbox;
    F.L = d_L;
    F.off = d_off;
    F.vb0 = d_vb0;
    F.gb0 = d_gb0;
    F.poff = d_poff;
    F.qf = d_qf;
    F.vbox = d_vbox;
    F.gbox = d_gbox;
    return F;
  }
  FinePools pools() const {
    FinePools p;
    for (int d = 0; d < 3; ++d) p.flx[d] = flx1[d];
    return p;
  }
  CoarseMap cmap() const {
    CoarseMap m;
    m.cmap = d_cmap;
    m.bmap = d_bmap;
    for (int d = 0; d < 3; ++d) {
      m.dlo[d] = Lc.dlo[d];
      m.n[d] = Lc.dhi[d] - Lc.dlo[d] + 1;
    }
    return m;
  }
  FluxRegDev reg() const {
    FluxRegDev r;
    r.nbnd = nbnd;
    r.cell = d_bcell;
    r.mask = d_mask;
    r.cstart = d_cstart;
    r.contrib = d_contrib;
    r.d = d_reg;
    r.cfp = d_cfp;
    return r;
  }
};

namespace {

inline unsigned blocks_of(int64_t n) { return unsigned((n + kBlk - 1) / kBlk); }

cudaError_t amr_issue_step(camr_amr* a, bool first, bool est = false) {
  cudaStream_t st = a->stream;
  const LGeom& Lc = a->Lc;
  const FineDev F = a->fine();
  const FinePools FP = a->pools();
  const CoarseMap CM = a->cmap();
  const FluxRegDev R = a->reg();
  const KParams& P = a->P;
  const bool mol = a->hp.do_mol != 0;
  const double fac = mol ? 0.5 : 1.0;
  const unsigned gv0 = blocks_of(a->ncell0);
  const int64_t npad0 = int64_t(Lc.pn[0]) * Lc.pn[1] * Lc.pn[2];
  const unsigned gf_valid = unsigned(a->h_vb0[a->nbox]);
  const unsigned gf_grown = unsigned(a->h_gb0[a->nbox]);
  const unsigned gf_interp = unsigned(a->h_ib0[a->nbox]);
  const unsigned gf_ilist =
      unsigned(std::max<int64_t>(1, (a->n_icell + kInterpItems - 1) / kInterpItems));
  const double* dt0 = &a->clock->dt0;
  const double* dt1 = &a->clock->dt1;
  DtCtl c{a->hp.cfl, a->hp.max_dt, a->hp.fixed_dt, a->hp.initial_dt, a->hp.init_shrink,
          a->hp.change_max};
  if (first || est) {
    k_reset_bits2<<<1, 1, 0, st>>>(a->bits0, a->bits1);
    k_est_dt<<<gv0, kBlk, 0, st>>>(Lc, P, a->S0, a->bits0);
    kf_est_dt<<<gf_valid, kBlk, 0, st>>>(F, P, a->S1, a->bits1);
    count_launch(3);
  }
  k_amr_dt<<<1, 1, 0, st>>>(c, first ? 1 : 0, a->bits0, a->bits1, a->clock, a->hist,
                            a->hist_cap);
  count_launch();
  cudaError_t e = cudaMemsetAsync(a->d_reg, 0, sizeof(double) * NVAR * std::max(a->nbnd, 1), st);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(a->d_cfp, 0, sizeof(double) * NVAR * std::max(a->nbnd, 1), st);
  if (e != cudaSuccess) return e;

  // ---- level 0: CAMR_advance with CrseAdd, no post_timestep yet ----
  // Each cleaning pass lists the cells below the density floor and a
  // one-block fixup resets them in the reference's order (a no-op launch
  // when the list is empty).
  const FloorList& fl = a->floor;
  FloorArgs fa{};
  fa.in = a->S0;
  fa.out = a->S0_old;
  k_clean_copy<<<gv0, kBlk, 0, st>>>(Lc, P, a->S0, a->S0_old, a->err, fl);
  k_floor_fixup<FLOOR_CLEAN><<<1, 1024, kFloorSmem, st>>>(Lc, P, fl, fa, a->err);
  fa.in = a->S0_old;
  fa.out = a->B0;
  k_expand<<<blocks_of(npad0), kBlk, 0, st>>>(Lc, P, a->S0_old, a->B0, a->err, fl);
  k_floor_fixup<FLOOR_EXPAND><<<1, 1024, kFloorSmem, st>>>(Lc, P, fl, fa, a->err);
  count_launch(2);
  count_launch(2);
  HydroLaunch H;
  for (int d = 0; d < 3; ++d) {
    H.g.lo[d] = Lc.dlo[d];
    H.g.hi[d] = Lc.dhi[d];
    H.g.dlo[d] = Lc.dlo[d];
    H.g.dhi[d] = Lc.dhi[d];
    H.g.bclo[d] = Lc.bclo[d];
    H.g.bchi[d] = Lc.bchi[d];
    H.g.dx[d] = Lc.dx[d];
  }
  H.P = P;
  H.has_src = false;
  H.mol = mol;
  H.dt = DtRef{0.0, dt0};
  H.err = a->err;
  auto sdfab = [&](double* p) {
    DFab f;
    f.p = p;
    for (int d = 0; d < 3; ++d) f.lo[d] = Lc.plo[d];
    f.sy = Lc.sy;
    f.sz = Lc.sz;
    f.sn = Lc.sn;
    return f;
  };
  for (int d = 0; d < 3; ++d) H.flx[d] = sdfab(a->flx0[d]);
  H.dsdt = sdfab(nullptr);
  FluxPtrs fp0;
  for (int d = 0; d < 3; ++d) {
    fp0.f[d] = a->flx0[d];
    fp0.q[d] = a->w0.qf[d];
  }
  const Space& sp0 = a->w0.s;
  const double vol0 = Lc.dx[0] * Lc.dx[1] * Lc.dx[2];
  const unsigned gb = blocks_of(std::max(a->nbnd, 1));
  H.uin = sdfab(a->B0);
  H.src = H.uin;
  e = launch_hydro_fluxes(H, a->w0, st);
  if (e != cudaSuccess) return e;
  k_crse_add<<<gb, kBlk, 0, st>>>(R, Lc, a->flx0[0], a->flx0[1], a->flx0[2], dt0, fac, vol0);
  count_launch();
  if (!mol) {
    k_update_ctu<<<gv0, kBlk, 0, st>>>(Lc, sp0, P, dt0, a->B0, a->S0_old, fp0, a->S0, nullptr,
                                       a->err, 0, fl);
    FloorArgs fu{nullptr, a->S0, a->B0, a->S0_old, fp0, sp0, dt0, nullptr, 0};
    k_floor_fixup<FLOOR_CTU><<<1, 1024, kFloorSmem, st>>>(Lc, P, fl, fu, a->err);
    count_launch();
    count_launch();
  } else {
    k_update_mol1<<<gv0, kBlk, 0, st>>>(Lc, sp0, P, dt0, a->B0, a->S0_old, fp0, a->S0);
    fa.in = a->S0;
    fa.out = a->B0_2;
    k_expand<<<blocks_of(npad0), kBlk, 0, st>>>(Lc, P, a->S0, a->B0_2, a->err, fl);
    k_floor_fixup<FLOOR_EXPAND><<<1, 1024, kFloorSmem, st>>>(Lc, P, fl, fa, a->err);
    count_launch();
    count_launch(2);
    H.uin = sdfab(a->B0_2);
    H.src = H.uin;
    e = launch_hydro_fluxes(H, a->w0, st);
    if (e != cudaSuccess) return e;
    k_crse_add<<<gb, kBlk, 0, st>>>(R, Lc, a->flx0[0], a->flx0[1], a->flx0[2], dt0, fac, vol0);
    k_update_mol2<<<gv0, kBlk, 0, st>>>(Lc, sp0, P, dt0, a->B0_2, a->S0_old, fp0, a->S0,
                                        nullptr, a->err, 0, fl);
    FloorArgs fu{nullptr, a->S0, a->B0_2, a->S0_old, fp0, sp0, dt0, nullptr, 0};
    k_floor_fixup<FLOOR_MOL2><<<1, 1024, kFloorSmem, st>>>(Lc, P, fl, fu, a->err);
    count_launch();
    count_launch(2);
  }

  // ---- level 1: two substeps ----
  const double volf8 = (F.nbox ? (Lc.dx[0] / RR) * (Lc.dx[1] / RR) * (Lc.dx[2] / RR) : 1.0) *
                       double(RR * RR * RR);
  const int3 fdlo = make_int3(a->fdlo[0], a->fdlo[1], a->fdlo[2]);
  const int3 fdn = make_int3(a->fdn[0], a->fdn[1], a->fdn[2]);
  for (int sc = 0; sc < RR; ++sc) {
    unsigned long long* fbits = (sc == RR - 1) ? a->bits1 : nullptr;
    k_fine_clock<<<1, 1, 0, st>>>(a->clock);
    FineFloorArgs ff{};
    ff.fp = FP;
    ff.dtp = dt1;
    ff.fdlo = fdlo;
    ff.fdn = fdn;
    ff.in = a->S1;
    ff.out = a->S1_old;
    kf_clean_copy<<<gf_valid, kBlk, 0, st>>>(F, P, a->S1, a->S1_old, a->err, fl);
    kf_floor_fixup<FFLOOR_CLEAN><<<1, 1024, kFloorSmem, st>>>(F, P, fl, ff, a->err);
    ff.in = a->S1_old;
    ff.out = a->B1;
    kf_fill<<<gf_grown, kBlk, 0, st>>>(F, P, CM, a->S1_old, a->B1, fdlo, fdn, a->err, fl);
    kf_floor_fixup<FFLOOR_FILL><<<1, 1024, kFloorSmem, st>>>(F, P, fl, ff, a->err);
    count_launch(2);
#if CAMR_INTERP_LIST
    kf_interp_list<<<gf_ilist, kBlk, 0, st>>>(F, P, Lc, a->S0_old, a->S0, &a->clock->ct[0],
                                              a->d_icell, a->n_icell, a->B1);
#else
    kf_interp<<<gf_interp, kBlk, 0, st>>>(F, P, CM, Lc, a->S0_old, a->S0, &a->clock->ct[0],
                                          a->d_ib0, a->B1);
#endif
    count_launch(4);
    camr_status cs = camr_batch_run(a->plan, 0.0, dt1, a->fine_mode, st);
    if (cs != CAMR_OK) return cudaErrorLaunchFailure;
    k_fine_add<<<gb, kBlk, 0, st>>>(R, F, FP, dt1, fac, volf8);
    count_launch();
    if (!mol) {
      kf_update_ctu<<<gf_valid, kBlk, 0, st>>>(F, FP, P, dt1, a->B1, a->S1_old, a->S1, fbits,
                                               a->err, fl);
      ff.in = nullptr;
      ff.out = a->S1;
      ff.B = a->B1;
      ff.S_old = a->S1_old;
      ff.bits = fbits;
      kf_floor_fixup<FFLOOR_CTU><<<1, 1024, kFloorSmem, st>>>(F, P, fl, ff, a->err);
      count_launch();
      count_launch();
    } else {
      kf_update_mol1<<<gf_valid, kBlk, 0, st>>>(F, FP, P, dt1, a->B1, a->S1_old, a->S1);
      // Sborder of the second stage reuses B1 (the first one is consumed)
      ff.in = a->S1;
      ff.out = a->B1;
      kf_fill<<<gf_grown, kBlk, 0, st>>>(F, P, CM, a->S1, a->B1, fdlo, fdn, a->err, fl);
      kf_floor_fixup<FFLOOR_FILL><<<1, 1024, kFloorSmem, st>>>(F, P, fl, ff, a->err);
      count_launch();
#if CAMR_INTERP_LIST
      kf_interp_list<<<gf_ilist, kBlk, 0, st>>>(F, P, Lc, a->S0_old, a->S0, &a->clock->ct[1],
                                                a->d_icell, a->n_icell, a->B1);
#else
      kf_interp<<<gf_interp, kBlk, 0, st>>>(F, P, CM, Lc, a->S0_old, a->S0, &a->clock->ct[1],
                                            a->d_ib0, a->B1);
#endif
      count_launch(3);
      cs = camr_batch_run(a->plan, 0.0, dt1, a->fine_mode, st);
      if (cs != CAMR_OK) return cudaErrorLaunchFailure;
      k_fine_add<<<gb, kBlk, 0, st>>>(R, F, FP, dt1, fac, volf8);
      kf_update_mol2<<<gf_valid, kBlk, 0, st>>>(F, FP, P, dt1, a->B1, a->S1_old, a->S1, fbits,
                                                a->err, fl);
      ff.in = nullptr;
      ff.out = a->S1;
      ff.B = a->B1;
      ff.S_old = a->S1_old;
      ff.bits = fbits;
      kf_floor_fixup<FFLOOR_MOL2><<<1, 1024, kFloorSmem, st>>>(F, P, fl, ff, a->err);
      count_launch();
      count_launch(2);
    }
  }

  // ---- level 0 post_timestep: reflux, avgDown, clean_state ----
  k_coarse_raw<<<gv0, kBlk, 0, st>>>(Lc, P, CM, R, F, a->S1, a->S0, fl);
  fa.in = a->S0;
  fa.out = a->S0;
  k_floor_fixup<FLOOR_INPLACE><<<1, 1024, kFloorSmem, st>>>(Lc, P, fl, fa, a->err);
  k_coarse_finish<<<gv0, kBlk, 0, st>>>(Lc, P, a->S0, a->bits0, a->err);
  count_launch(3);
  return cudaGetLastError();
}

void amr_free(camr_amr* a) {
  if (a->graph_ready) cudaGraphExecDestroy(a->graph);
  if (a->plan) camr_batch_destroy(a->plan);
  void* ptrs[] = {a->S0, a->S0_old, a->B0, a->B0_2, a->flx0[0], a->flx0[1], a->flx0[2],
                  a->work0, a->S1, a->S1_old, a->B1, a->flx1[0], a->flx1[1], a->flx1[2],
                  a->d_L, a->d_off, a->d_vb0, a->d_gb0, a->d_ib0, a->d_poff, a->d_qf, a->d_cmap,
                  a->d_bmap, a->d_bcell, a->d_mask, a->d_cstart, a->d_contrib, a->d_reg,
                  a->d_cfp, a->clock, a->hist, a->bits0, a->bits1, a->err, a->staging0,
                  a->staging1, a->floor.count, a->floor.cells, a->floor.enforced,
                  a->floor.total, a->d_icell, a->d_vbox, a->d_gbox};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (a->own_stream) cudaStreamDestroy(a->stream);
  delete a;
}

}  // namespace

extern "C" {

camr_status camr_amr_create(const camr_level_desc* base, int nbox, const int* boxes,
                            const camr_hydro_params* p, void* stream, camr_amr** out) {
  if (!base || !p || !out || nbox < 1 || !boxes) return CAMR_ERR_INVALID;
  if (p->riemann_solver < 0 || p->riemann_solver > 1) return CAMR_ERR_UNSUPPORTED;
  if (!p->do_mol && p->ppm_type != 0 && p->ppm_type != 1) return CAMR_ERR_INVALID;
  if (p->cfl <= 0.0 || p->cfl > 1.0) return CAMR_ERR_INVALID;
  if (p->do_mol && p->cfl > 0.3 && p->fixed_dt <= 0.0) return CAMR_ERR_INVALID;
  if (p->add_grav_src && p->const_grav != 0.0 && !p->do_mol) return CAMR_ERR_UNSUPPORTED;
  const camr_geom& g = base->geom;
  for (int d = 0; d < 3; ++d) {
    if (!g.is_periodic[d]) return CAMR_ERR_UNSUPPORTED;
    if (g.dom_hi[d] < g.dom_lo[d]) return CAMR_ERR_INVALID;
  }
  // fine boxes: coarse-aligned, inside the fine domain, disjoint
  const int cn[3] = {g.dom_hi[0] - g.dom_lo[0] + 1, g.dom_hi[1] - g.dom_lo[1] + 1,
                     g.dom_hi[2] - g.dom_lo[2] + 1};
  const int64_t ncell0 = int64_t(cn[0]) * cn[1] * cn[2];
  std::vector<int> cmap(ncell0, -1);
  auto cidx = [&](int i, int j, int k) {
    const int c[3] = {i, j, k};
    int w[3];
    for (int d = 0; d < 3; ++d) w[d] = (((c[d] - g.dom_lo[d]) % cn[d]) + cn[d]) % cn[d];
    return int64_t(w[0]) + int64_t(cn[0]) * (w[1] + int64_t(cn[1]) * w[2]);
  };
  for (int b = 0; b < nbox; ++b) {
    const int* bx = boxes + 6 * b;
    for (int d = 0; d < 3; ++d) {
      const int lo = bx[d], hi = bx[3 + d];
      if (hi < lo || (lo % 2) != 0 || (hi % 2) != 1 || lo < RR * g.dom_lo[d] ||
          hi > RR * g.dom_hi[d] + 1)
        return CAMR_ERR_INVALID;
    }
    for (int k = bx[2] / 2; k <= bx[5] / 2; ++k)
      for (int j = bx[1] / 2; j <= bx[4] / 2; ++j)
        for (int i = bx[0] / 2; i <= bx[3] / 2; ++i) {
          int64_t c = cidx(i, j, k);
          if (cmap[c] >= 0) return CAMR_ERR_INVALID;  // overlap
          cmap[c] = b;
        }
  }
  if (kf_floor_prepare() != cudaSuccess) return CAMR_ERR_CUDA;
  camr_amr* a = new (std::nothrow) camr_amr();
  if (!a) return CAMR_ERR_NOMEM;
  a->hp = *p;
  a->P = make_kparams(*p);
  a->desc = *base;
  a->stream = static_cast<cudaStream_t>(stream);
  if (!a->stream) {
    if (cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete a;
      return CAMR_ERR_CUDA;
    }
    a->own_stream = true;
  }
  cudaStream_t st = a->stream;
  // ---- level 0 geometry and arrays ----
  LGeom& Lc = a->Lc;
  for (int d = 0; d < 3; ++d) {
    Lc.dlo[d] = g.dom_lo[d];
    Lc.dhi[d] = g.dom_hi[d];
    Lc.plo[d] = g.dom_lo[d] - NGROW;
    Lc.pn[d] = cn[d] + 2 * NGROW;
    Lc.periodic[d] = 1;
    Lc.bclo[d] = g.bc_lo[d];
    Lc.bchi[d] = g.bc_hi[d];
    Lc.dx[d] = g.dx[d];
    Lc.boxsz[d] = base->max_grid_size[d] > 0 ? base->max_grid_size[d] : cn[d];
  }
  const Space sp0 = make_space(Lc.dlo, Lc.dhi);
  Lc.sy = sp0.sy;
  Lc.sz = sp0.sz;
  Lc.sn = sp0.sn;
  lgeom_finish(Lc);
  a->ncell0 = ncell0;
  const bool mol = p->do_mol != 0;
  cudaError_t e = cudaSuccess;
  auto alloc = [&](void** ptr, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(ptr, std::max<size_t>(bytes, 8));
    if (e == cudaSuccess) e = cudaMemsetAsync(*ptr, 0, std::max<size_t>(bytes, 8), st);
  };
  const size_t sbytes0 = size_t(sp0.sn) * NVAR * sizeof(double);
  alloc(reinterpret_cast<void**>(&a->S0), sbytes0);
  alloc(reinterpret_cast<void**>(&a->S0_old), sbytes0);
  alloc(reinterpret_cast<void**>(&a->B0), sbytes0);
  if (mol) alloc(reinterpret_cast<void**>(&a->B0_2), sbytes0);
  for (int d = 0; d < 3; ++d) alloc(reinterpret_cast<void**>(&a->flx0[d]), sbytes0);
  alloc(reinterpret_cast<void**>(&a->work0), work_doubles(sp0, mol, false) * sizeof(double));
  alloc(reinterpret_cast<void**>(&a->staging0), size_t(ncell0) * NVAR * sizeof(double));
  // ---- level 1 ----
  a->nbox = nbox;
  for (int d = 0; d < 3; ++d) {
    a->fdlo[d] = RR * g.dom_lo[d];
    a->fdn[d] = RR * cn[d];
  }
  std::vector<LGeom> hL(nbox);
  std::vector<int64_t> off(nbox), poff(nbox);
  a->h_vb0.assign(nbox + 1, 0);
  a->h_gb0.assign(nbox + 1, 0);
  a->h_ib0.assign(nbox + 1, 0);
  int64_t total = 0, ptotal = 0;
  for (int b = 0; b < nbox; ++b) {
    const int* bx = boxes + 6 * b;
    LGeom& L = hL[b];
    int lo[3], hi[3];
    int64_t nv = 1, ng = 1;
    for (int d = 0; d < 3; ++d) {
      lo[d] = bx[d];
      hi[d] = bx[3 + d];
      L.dlo[d] = lo[d];
      L.dhi[d] = hi[d];
      L.plo[d] = lo[d] - NGROW;
      L.pn[d] = hi[d] - lo[d] + 1 + 2 * NGROW;
      L.periodic[d] = 0;
      L.bclo[d] = 0;
      L.bchi[d] = 0;
      L.dx[d] = g.dx[d] / RR;
      L.boxsz[d] = hi[d] - lo[d] + 1;
      nv *= hi[d] - lo[d] + 1;
      ng *= L.pn[d];
    }
    const Space sp = make_space(lo, hi);
    L.sy = sp.sy;
    L.sz = sp.sz;
    L.sn = sp.sn;
    lgeom_finish(L);
    off[b] = total;
    total += (int64_t(sp.sn) * NVAR + 31) / 32 * 32;
    poff[b] = ptotal;
    ptotal += nv * NVAR;
    a->ncell1 += nv;
    a->h_vb0[b + 1] = a->h_vb0[b] + (nv + kBlk - 1) / kBlk;
    a->h_gb0[b + 1] = a->h_gb0[b] + (ng + kBlk - 1) / kBlk;
    int64_t nci = 1;  // coarse cells of grow(coarsened box, 2)
    for (int d = 0; d < 3; ++d) nci *= (hi[d] - lo[d] + 1) / RR + 4;
    a->h_ib0[b + 1] = a->h_ib0[b] + (nci + kBlk - 1) / kBlk;
  }
  a->pool = total;
  const size_t pbytes = size_t(total) * sizeof(double);
  alloc(reinterpret_cast<void**>(&a->S1), pbytes);
  alloc(reinterpret_cast<void**>(&a->S1_old), pbytes);
  alloc(reinterpret_cast<void**>(&a->B1), pbytes);
  for (int d = 0; d < 3; ++d) alloc(reinterpret_cast<void**>(&a->flx1[d]), pbytes);
  alloc(reinterpret_cast<void**>(&a->staging1), size_t(ptotal) * sizeof(double));
  alloc(reinterpret_cast<void**>(&a->clock), sizeof(AmrClock));
  alloc(reinterpret_cast<void**>(&a->hist), sizeof(double) * 2 * a->hist_cap);
  alloc(reinterpret_cast<void**>(&a->bits0), sizeof(unsigned long long));
  alloc(reinterpret_cast<void**>(&a->bits1), sizeof(unsigned long long));
  alloc(reinterpret_cast<void**>(&a->err), sizeof(DevError));
  alloc(reinterpret_cast<void**>(&a->floor.count), sizeof(int));
  alloc(reinterpret_cast<void**>(&a->floor.cells), sizeof(int64_t) * kFloorCap);
  alloc(reinterpret_cast<void**>(&a->floor.enforced), sizeof(double) * NVAR * kFloorCap);
  alloc(reinterpret_cast<void**>(&a->floor.total), sizeof(unsigned long long));
  if (e != cudaSuccess) {
    amr_free(a);
    return CAMR_ERR_NOMEM;
  }
  if (e == cudaSuccess) e = upload(&a->d_L, hL, st);
  if (e == cudaSuccess) e = upload(&a->d_off, off, st);
  if (e == cudaSuccess) e = upload(&a->d_poff, poff, st);
  if (e == cudaSuccess) e = upload(&a->d_vb0, a->h_vb0, st);
  if (e == cudaSuccess) e = upload(&a->d_gb0, a->h_gb0, st);
  if (e == cudaSuccess) e = upload(&a->d_ib0, a->h_ib0, st);
  if (CAMR_FINE_BLOCKMAP) {
    // the box of every block of the valid-cell and grown-cell launches, so
    // that a block reads it instead of binary-searching vb0 / gb0
    auto block_boxes = [&](const std::vector<int64_t>& b0, int** dst) {
      std::vector<int> m(size_t(b0[size_t(nbox)]), 0);
      for (int b = 0; b < nbox; ++b)
        for (int64_t q = b0[size_t(b)]; q < b0[size_t(b) + 1]; ++q) m[size_t(q)] = b;
      if (e == cudaSuccess && !m.empty()) e = upload(dst, m, st);
    };
    block_boxes(a->h_vb0, &a->d_vbox);
    block_boxes(a->h_gb0, &a->d_gbox);
  }
  {
    // the coarse cells of grow(coarsened box, 2) outside the coarsened box
    // that no fine box covers, in kf_interp's order
    std::vector<int4> icell;
    for (int b = 0; b < nbox; ++b) {
      const int* bx = boxes + 6 * b;
      int clo[3], ncn[3];
      for (int d = 0; d < 3; ++d) {
        clo[d] = bx[d] / RR - 2;
        ncn[d] = (bx[3 + d] - bx[d] + 1) / RR + 4;
      }
      for (int kk = 0; kk < ncn[2]; ++kk)
        for (int jj = 0; jj < ncn[1]; ++jj)
          for (int ii = 0; ii < ncn[0]; ++ii) {
            if (ii >= 2 && ii < ncn[0] - 2 && jj >= 2 && jj < ncn[1] - 2 && kk >= 2 &&
                kk < ncn[2] - 2)
              continue;
            const int ci = clo[0] + ii, cj = clo[1] + jj, ck = clo[2] + kk;
            if (cmap[cidx(ci, cj, ck)] >= 0) continue;
            icell.push_back(make_int4(b, ci, cj, ck));
          }
    }
    a->n_icell = int64_t(icell.size());
    if (e == cudaSuccess && !icell.empty()) e = upload(&a->d_icell, icell, st);
  }
  // the fine hydro plan (fluxes only) over the B1 pool
  std::vector<camr_box_task> tasks(nbox);
  for (int b = 0; b < nbox; ++b) {
    camr_box_task& t = tasks[b];
    std::memset(&t, 0, sizeof(t));
    const LGeom& L = hL[b];
    auto fab = [&](double* base_ptr) {
      camr_fab f{};
      f.ptr = base_ptr + off[b];
      for (int d = 0; d < 3; ++d) {
        f.lo[d] = L.plo[d];
        f.hi[d] = L.dhi[d] + NGROW + 1;
      }
      f.jstride = L.sy;
      f.kstride = L.sz;
      f.nstride = L.sn;
      f.ncomp = NVAR;
      return f;
    };
    for (int d = 0; d < 3; ++d) {
      t.lo[d] = L.dlo[d];
      t.hi[d] = L.dhi[d];
    }
    t.uin = fab(a->B1);
    for (int d = 0; d < 3; ++d) t.flx[d] = fab(a->flx1[d]);
  }
  camr_geom fg{};
  for (int d = 0; d < 3; ++d) {
    fg.dom_lo[d] = a->fdlo[d];
    fg.dom_hi[d] = a->fdlo[d] + a->fdn[d] - 1;
    fg.is_periodic[d] = 1;
    fg.bc_lo[d] = g.bc_lo[d];
    fg.bc_hi[d] = g.bc_hi[d];
    fg.dx[d] = g.dx[d] / RR;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    amr_free(a);
    return CAMR_ERR_CUDA;
  }
  camr_status cs = batch_create_fluxes(nbox, tasks.data(), &fg, p, st, &a->plan);
  if (cs != CAMR_OK) {
    amr_free(a);
    return cs;
  }
  std::vector<double*> qf(size_t(nbox) * 3);
  for (int b = 0; b < nbox; ++b)
    for (int d = 0; d < 3; ++d) qf[3 * b + d] = batch_work(a->plan, b).qf[d];
  e = upload(&a->d_qf, qf, st);
  // ---- flux register: boundary cells, masks, FineAdd contribution lists ----
  std::vector<int> bmap(ncell0, -1), bcell, mask;
  for (int k = 0; k < cn[2]; ++k)
    for (int j = 0; j < cn[1]; ++j)
      for (int i = 0; i < cn[0]; ++i) {
        const int ci = g.dom_lo[0] + i, cj = g.dom_lo[1] + j, ck = g.dom_lo[2] + k;
        const int64_t c = cidx(ci, cj, ck);
        if (cmap[c] >= 0) continue;
        int m = 0;
        const int cc[3] = {ci, cj, ck};
        for (int d = 0; d < 3; ++d) {
          int lo3[3] = {cc[0], cc[1], cc[2]}, hi3[3] = {cc[0], cc[1], cc[2]};
          lo3[d] -= 1;
          hi3[d] += 1;
          if (cmap[cidx(lo3[0], lo3[1], lo3[2])] >= 0) m |= 1 << (2 * d);
          if (cmap[cidx(hi3[0], hi3[1], hi3[2])] >= 0) m |= 1 << (2 * d + 1);
        }
        if (m) {
          bmap[c] = int(mask.size());
          mask.push_back(m);
          bcell.push_back(ci);
          bcell.push_back(cj);
          bcell.push_back(ck);
        }
      }
  a->nbnd = int(mask.size());
  // contributions in FineAdd's order: box, direction, low side then high
  std::vector<std::vector<int4>> per(a->nbnd);
  for (int b = 0; b < nbox; ++b) {
    const int* bx = boxes + 6 * b;
    int clo[3], chi[3];
    for (int d = 0; d < 3; ++d) {
      clo[d] = bx[d] / RR;
      chi[d] = bx[3 + d] / RR;
    }
    for (int d = 0; d < 3; ++d)
      for (int side = 0; side < 2; ++side) {
        int lo3[3] = {clo[0], clo[1], clo[2]}, hi3[3] = {chi[0], chi[1], chi[2]};
        lo3[d] = hi3[d] = side ? chi[d] + 1 : clo[d] - 1;
        for (int k = lo3[2]; k <= hi3[2]; ++k)
          for (int j = lo3[1]; j <= hi3[1]; ++j)
            for (int i = lo3[0]; i <= hi3[0]; ++i) {
              const int64_t c = cidx(i, j, k);
              if (cmap[c] >= 0) continue;
              per[bmap[c]].push_back(make_int4(b, d, side, 0));
            }
      }
  }
  std::vector<int> cstart(a->nbnd + 1, 0);
  std::vector<int4> contrib;
  for (int c = 0; c < a->nbnd; ++c) {
    cstart[c] = int(contrib.size());
    contrib.insert(contrib.end(), per[c].begin(), per[c].end());
  }
  cstart[a->nbnd] = int(contrib.size());
  if (e == cudaSuccess) e = upload(&a->d_cmap, cmap, st);
  if (e == cudaSuccess) e = upload(&a->d_bmap, bmap, st);
  if (e == cudaSuccess) e = upload(&a->d_bcell, bcell, st);
  if (e == cudaSuccess) e = upload(&a->d_mask, mask, st);
  if (e == cudaSuccess) e = upload(&a->d_cstart, cstart, st);
  if (e == cudaSuccess) e = upload(&a->d_contrib, contrib, st);
  alloc(reinterpret_cast<void**>(&a->d_reg), sizeof(double) * NVAR * std::max(a->nbnd, 1));
  alloc(reinterpret_cast<void**>(&a->d_cfp), sizeof(double) * NVAR * std::max(a->nbnd, 1));
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    amr_free(a);
    return CAMR_ERR_CUDA;
  }
  a->w0.s = sp0;
  work_carve(a->w0, a->work0, mol, false);
  *out = a;
  return CAMR_OK;
}

camr_status camr_amr_destroy(camr_amr* a) {
  if (!a) return CAMR_ERR_INVALID;
  amr_free(a);
  return CAMR_OK;
}

camr_status camr_amr_set_state(camr_amr* a, const double* S0, const double* S1, int host) {
  if (!a || !S0 || !S1) return CAMR_ERR_INVALID;
  const cudaMemcpyKind kind = host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  cudaError_t e = cudaMemcpyAsync(a->staging0, S0, size_t(a->ncell0) * NVAR * sizeof(double),
                                  kind, a->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(a->staging1, S1, size_t(a->ncell1) * NVAR * sizeof(double), kind,
                        a->stream);
  if (e != cudaSuccess) return CAMR_ERR_CUDA;
  k_pack<<<blocks_of(a->ncell0), kBlk, 0, a->stream>>>(a->Lc, a->S0, a->staging0, 0);
  kf_pack<<<unsigned(a->h_vb0[a->nbox]), kBlk, 0, a->stream>>>(a->fine(), a->S1, a->staging1, 0);
  count_launch(2);
  e = cudaMemsetAsync(a->clock, 0, sizeof(AmrClock), a->stream);
  a->steps_taken = 0;
  a->restart_est = false;
  if (e != cudaSuccess) return CAMR_ERR_CUDA;
  return cuda_status_of(cudaGetLastError());
}

camr_status camr_amr_get_state(camr_amr* a, double* S0, double* S1, int host) {
  if (!a || !S0 || !S1) return CAMR_ERR_INVALID;
  k_pack<<<blocks_of(a->ncell0), kBlk, 0, a->stream>>>(a->Lc, a->S0, a->staging0, 1);
  kf_pack<<<unsigned(a->h_vb0[a->nbox]), kBlk, 0, a->stream>>>(a->fine(), a->S1, a->staging1, 1);
  count_launch(2);
  const cudaMemcpyKind kind = host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  cudaError_t e = cudaMemcpyAsync(S0, a->staging0, size_t(a->ncell0) * NVAR * sizeof(double),
                                  kind, a->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(S1, a->staging1, size_t(a->ncell1) * NVAR * sizeof(double), kind,
                        a->stream);
  if (e == cudaSuccess && host) e = cudaStreamSynchronize(a->stream);
  return cuda_status_of(e);
}

camr_status camr_amr_init_finalize(camr_amr* a) {
  if (!a) return CAMR_ERR_INVALID;
  k_init_finalize<<<blocks_of(a->ncell0), kBlk, 0, a->stream>>>(a->Lc, a->P, a->S0);
  kf_init_finalize<<<unsigned(a->h_vb0[a->nbox]), kBlk, 0, a->stream>>>(a->fine(), a->P, a->S1);
  k_init_avgdown<<<blocks_of(a->ncell0), kBlk, 0, a->stream>>>(a->Lc, a->cmap(), a->fine(),
                                                              a->S1, a->S0);
  count_launch(3);
  return cuda_status_of(cudaGetLastError());
}

camr_status camr_amr_advance(camr_amr* a, int nsteps) {
  if (!a || nsteps < 0) return CAMR_ERR_INVALID;
  for (int s = 0; s < nsteps; ++s) {
    const bool first = a->steps_taken == 0;
    cudaError_t e;
    if (a->restart_est) {
      a->restart_est = false;
      e = amr_issue_step(a, false, true);
    } else if (!first && a->desc.use_graph && a->fine_mode == CAMR_BATCH_PERSISTENT) {
      if (!a->graph_ready) {
        cudaGraph_t gr;
        e = cudaStreamBeginCapture(a->stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return cuda_status_of(e);
        const int64_t before = launches_now();
        cudaError_t e1 = amr_issue_step(a, false);
        a->kernels_per_step = launches_now() - before;
        launches_sub(a->kernels_per_step);
        e = cudaStreamEndCapture(a->stream, &gr);
        if (e1 != cudaSuccess) return cuda_status_of(e1);
        if (e != cudaSuccess) return cuda_status_of(e);
        e = cudaGraphInstantiate(&a->graph, gr, 0);
        cudaGraphDestroy(gr);
        if (e != cudaSuccess) return cuda_status_of(e);
        a->graph_ready = true;
      }
      e = cudaGraphLaunch(a->graph, a->stream);
      count_launch(int(a->kernels_per_step));
    } else {
      e = amr_issue_step(a, first);
    }
    if (e != cudaSuccess) return cuda_status_of(e);
    a->steps_taken++;
  }
  return CAMR_OK;
}

camr_status camr_amr_restart(camr_amr* a, const double clock[4], int steps_done) {
  if (!a || !clock || steps_done < 1 || !(clock[2] > 0.0) || !(clock[3] > 0.0))
    return CAMR_ERR_INVALID;
  AmrClock h;
  cudaError_t e = cudaMemcpyAsync(&h, a->clock, sizeof(h), cudaMemcpyDeviceToHost, a->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(a->stream);
  if (e != cudaSuccess) return cuda_status_of(e);
  h.tc_new = clock[0];
  h.tf_new = clock[1];
  h.dt0 = clock[2];
  h.dt1 = clock[3];
  e = cudaMemcpyAsync(a->clock, &h, sizeof(h), cudaMemcpyHostToDevice, a->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(a->stream);
  if (e != cudaSuccess) return cuda_status_of(e);
  a->steps_taken = steps_done;
  a->restart_est = true;
  return CAMR_OK;
}

camr_status camr_amr_floor_resets(camr_amr* a, int64_t* cells) {
  if (!a || !cells) return CAMR_ERR_INVALID;
  unsigned long long h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, a->floor.total, sizeof(h), cudaMemcpyDeviceToHost,
                                  a->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(a->stream);
  if (e != cudaSuccess) return cuda_status_of(e);
  *cells = int64_t(h);
  return CAMR_OK;
}

camr_status camr_amr_clock(camr_amr* a, double clock[4]) {
  if (!a || !clock) return CAMR_ERR_INVALID;
  AmrClock h;
  cudaError_t e = cudaMemcpyAsync(&h, a->clock, sizeof(h), cudaMemcpyDeviceToHost, a->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(a->stream);
  if (e != cudaSuccess) return cuda_status_of(e);
  clock[0] = h.tc_new;
  clock[1] = h.tf_new;
  clock[2] = h.dt0;
  clock[3] = h.dt1;
  return CAMR_OK;
}

camr_status camr_amr_autotune(camr_amr* a) {
  if (!a || a->steps_taken == 0) return CAMR_ERR_INVALID;
  AmrClock h;
  cudaError_t e = cudaMemcpyAsync(&h, a->clock, sizeof(h), cudaMemcpyDeviceToHost, a->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(a->stream);
  if (e != cudaSuccess) return cuda_status_of(e);
  // the captured graph holds the old launch shapes
  if (a->graph_ready) {
    cudaGraphExecDestroy(a->graph);
    a->graph_ready = false;
  }
  return camr_batch_autotune(a->plan, h.dt1, a->stream);
}

camr_status camr_amr_set_fine_mode(camr_amr* a, int mode) {
  if (!a || (mode != CAMR_BATCH_PERSISTENT && mode != CAMR_BATCH_PER_BOX)) return CAMR_ERR_INVALID;
  a->fine_mode = mode;
  return CAMR_OK;
}

int64_t camr_amr_fine_cells(camr_amr* a) { return a ? a->ncell1 : 0; }
int64_t camr_amr_kernels_per_step(camr_amr* a) { return a ? a->kernels_per_step : 0; }

camr_status camr_amr_stream(camr_amr* a, void** stream) {
  if (!a || !stream) return CAMR_ERR_INVALID;
  *stream = static_cast<void*>(a->stream);
  return CAMR_OK;
}

camr_status camr_amr_get_error(camr_amr* a, camr_error_info* info) {
  if (!a || !info) return CAMR_ERR_INVALID;
  DevError h;
  cudaError_t e = cudaMemcpyAsync(&h, a->err, sizeof(h), cudaMemcpyDeviceToHost, a->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(a->err, 0, sizeof(DevError), a->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(a->stream);
  if (e != cudaSuccess) return CAMR_ERR_CUDA;
  info->code = h.code;
  info->i = h.i;
  info->j = h.j;
  info->k = h.k;
  return h.code ? CAMR_ERR_NUMERIC : CAMR_OK;
}

}  // extern "C"
