// Fab-level pieces of the level step, for callers that keep their own box
// loop (a CAMR build whose AMReX level driver replaces only parts of the
// step): the single-level ghost fill of expand_state's FillPatch, clean_state
// and estTimeStep over a list of boxes held as fabs, and the library-wide
// device error word that the per-box entry points report into.
//
//   camr_fill_ghosts   FillPatch on one level (Source/CAMR.cpp:1243-1250):
//                      FillBoundary (interior and periodic ghosts) + the BC
//                      fill of Source/Utils/BCfill.cpp:119-134 with the BC map
//                      of Source/Utils/CAMR_setup.cpp:19-21
//   camr_clean_state   clean_state (Source/CAMR.cpp:1253-1262)
//   camr_est_dt        estTimeStep's hydro limit (Source/CAMR.cpp:490-563,
//                      Source/Utils/Timestep.H:18-61)
//   camr_get_error     the device error word (first failure wins)
#include <cuda_runtime.h>

#include <cfloat>
#include <cstring>
#include <mutex>
#include <vector>

#include "level_point.cuh"

namespace camr {
namespace {

// One box of the caller's list: its valid box, the region of its fab that
// the call touches (valid box grown by ng), and the fab.
struct FabBox {
  int lo[3], hi[3];
  int glo[3], ghi[3];
  DFab f;
};

struct FabSet {
  const FabBox* box;
  int nbox;
  int dlo[3], dhi[3];
  int periodic[3], bclo[3], bchi[3];
  double dx[3];
};

constexpr int kFB = 256;

// The library-wide error word of the per-box and fab-level calls.
static __device__ DevError g_lib_err;

constexpr int kMaxDevices = 64;
std::mutex g_err_mu;
DevError* g_err_addr[kMaxDevices] = {};

__device__ __forceinline__ bool in_box(const FabBox& b, int i, int j, int k) {
  return i >= b.lo[0] && i <= b.hi[0] && j >= b.lo[1] && j <= b.hi[1] && k >= b.lo[2] &&
         k <= b.hi[2];
}

// The box whose valid cells hold (i,j,k), or -1.  `hint` is tried first:
// the ghost cells a thread block fills mostly come from one neighbour.
__device__ __forceinline__ int find_owner(const FabSet& S, int i, int j, int k, int& hint) {
  if (hint >= 0 && in_box(S.box[hint], i, j, k)) return hint;
  for (int b = 0; b < S.nbox; ++b) {
    if (in_box(S.box[b], i, j, k)) {
      hint = b;
      return b;
    }
  }
  return -1;
}

// The cell of box blockIdx.y's fab region that thread t stands on.
__device__ __forceinline__ bool fab_region_cell(const FabBox& b, int64_t t, int& i, int& j,
                                                int& k) {
  const int n0 = b.ghi[0] - b.glo[0] + 1, n1 = b.ghi[1] - b.glo[1] + 1,
            n2 = b.ghi[2] - b.glo[2] + 1;
  if (t >= int64_t(n0) * n1 * n2) return false;
  const int64_t nxy = int64_t(n0) * n1;
  k = int(t / nxy);
  const int64_t r = t - int64_t(k) * nxy;
  j = int(r / n0);
  i = int(r - int64_t(j) * n0);
  i += b.glo[0];
  j += b.glo[1];
  k += b.glo[2];
  return true;
}

// Where a ghost cell takes its value from: its periodic image inside the
// domain and, past a physical boundary, the BC map's source cell
// (foextrap / ext_dir copy the boundary cell, as Exec/Sod's bcnormal does;
// reflect_even / reflect_odd mirror it).  neg_mask bit n: component n
// changes sign (reflect_odd).  physical: a physical boundary was crossed.
__device__ __forceinline__ void ghost_source(const FabSet& S, int i, int j, int k, int src[3],
                                             unsigned& neg_mask, bool& physical) {
  const int c[3] = {i, j, k};
  neg_mask = 0u;
  physical = false;
  for (int d = 0; d < 3; ++d) {
    src[d] = c[d];
    if (c[d] >= S.dlo[d] && c[d] <= S.dhi[d]) continue;
    if (S.periodic[d]) {
      const int len = S.dhi[d] - S.dlo[d] + 1;
      src[d] = S.dlo[d] + (((c[d] - S.dlo[d]) % len) + len) % len;
      continue;
    }
    physical = true;
    const bool low = c[d] < S.dlo[d];
    const int phys = low ? S.bclo[d] : S.bchi[d];
    // the source index is the same for every component of one BC word
    const int t = bc_kind(URHO, d, phys);
    if (t == 1 || t == 2) src[d] = low ? S.dlo[d] : S.dhi[d];
    else src[d] = low ? 2 * S.dlo[d] - c[d] - 1 : 2 * S.dhi[d] - c[d] + 1;
    for (int n = 0; n < NVAR; ++n)
      if (bc_kind(n, d, phys) == 4) neg_mask ^= 1u << n;
  }
}

// FillPatch on one level: every ghost cell of every fab (within ng) whose
// source cell is a valid cell of some box of the list.  Ghost cells whose
// source no box holds (a coarse-fine boundary) are left as they are.
__global__ void __launch_bounds__(kFB) k_fab_fill(FabSet S) {
  const FabBox& b = S.box[blockIdx.y];
  int i, j, k;
  if (!fab_region_cell(b, int64_t(blockIdx.x) * kFB + threadIdx.x, i, j, k)) return;
  if (in_box(b, i, j, k)) return;
  int src[3];
  unsigned neg;
  bool physical;
  ghost_source(S, i, j, k, src, neg, physical);
  int hint = -1;
  const int o = find_owner(S, src[0], src[1], src[2], hint);
  if (o < 0) return;
  const DFab& fo = S.box[o].f;
  for (int n = 0; n < NVAR; ++n) {
    const double v = fo(src[0], src[1], src[2], n);
    b.f(i, j, k, n) = ((neg >> n) & 1u) ? -v : v;
  }
}

// enforce_min_density, pass 1: list the valid cells below the floor, keyed
// by (box, raster position in the box).
__global__ void __launch_bounds__(kFB) k_fab_floor_list(FabSet S, KParams P, FloorList fl) {
  const FabBox& b = S.box[blockIdx.y];
  const int n0 = b.hi[0] - b.lo[0] + 1, n1 = b.hi[1] - b.lo[1] + 1, n2 = b.hi[2] - b.lo[2] + 1;
  const int64_t t = int64_t(blockIdx.x) * kFB + threadIdx.x;
  if (t >= int64_t(n0) * n1 * n2) return;
  const int64_t nxy = int64_t(n0) * n1;
  const int k = int(t / nxy);
  const int64_t r = t - int64_t(k) * nxy;
  const int j = int(r / n0);
  const int i = int(r - int64_t(j) * n0);
  if (b.f(b.lo[0] + i, b.lo[1] + j, b.lo[2] + k, URHO) < P.small_dens) {
    const int slot = atomicAdd(fl.count, 1);
    if (slot < kFloorCap) fl.cells[slot] = (int64_t(blockIdx.y) << 40) | t;
  }
}

// enforce_min_density, pass 2 (Source/CAMR.cpp:941-1045): the listed cells
// of each box in raster order, reset in place, so that a later cell sees
// an earlier reset exactly as the reference's sequential loop does.  Boxes
// are independent (the neighbour window is the cell's own box): one thread
// walks each box.  More than kFloorCap cells: error code 5, no reset.
__global__ void __launch_bounds__(1024) k_fab_floor_walk(FabSet S, KParams P, FloorList fl,
                                                          DevError* err) {
  constexpr int64_t kMask = (int64_t(1) << 40) - 1;
  extern __shared__ int64_t key[];
  const int n = *fl.count;
  if (n == 0) return;
  if (n > kFloorCap) {
    __syncthreads();
    if (threadIdx.x == 0) {
      const int64_t c = fl.cells[0];
      const FabBox& b = S.box[int(c >> 40)];
      report_error(err, 5, b.lo[0], b.lo[1], b.lo[2]);
      *fl.count = 0;
    }
    return;
  }
  int N = 1;
  while (N < n) N <<= 1;
  for (int t = threadIdx.x; t < N; t += blockDim.x) key[t] = (t < n) ? fl.cells[t] : INT64_MAX;
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
  for (int t0 = threadIdx.x; t0 < n; t0 += blockDim.x) {
    const int64_t boxid = key[t0] >> 40;
    if (t0 > 0 && (key[t0 - 1] >> 40) == boxid) continue;
    const FabBox& b = S.box[int(boxid)];
    const DFab& f = b.f;
    const int n0 = b.hi[0] - b.lo[0] + 1, n1 = b.hi[1] - b.lo[1] + 1;
    for (int m = t0; m < n && (key[m] >> 40) == boxid; ++m) {
      const int64_t t = key[m] & kMask;
      const int64_t nxy = int64_t(n0) * n1;
      const int k = b.lo[2] + int(t / nxy);
      const int64_t r = t - int64_t(k - b.lo[2]) * nxy;
      const int j = b.lo[1] + int(r / n0);
      const int i = b.lo[0] + int(r - int64_t(j - b.lo[1]) * n0);
      if (f(i, j, k, URHO) == 0.) {
        report_error(err, 3, i, j, k);  // amrex::Error in the reference
        continue;
      }
      double max_dens = f(i, j, k, URHO);
      int is = i, js = j, ks = k;
      for (int kk = -1; kk <= 1; kk++)
        for (int jj = -1; jj <= 1; jj++)
          for (int ii = -1; ii <= 1; ii++) {
            if (i + ii >= b.lo[0] && j + jj >= b.lo[1] && k + kk >= b.lo[2] &&
                i + ii <= b.hi[0] && j + jj <= b.hi[1] && k + kk <= b.hi[2]) {
              if (f(i + ii, j + jj, k + kk, URHO) > max_dens) {
                is = i + ii;
                js = j + jj;
                ks = k + kk;
                max_dens = f(is, js, ks, URHO);
              }
            }
          }
      if (max_dens < P.small_dens) {
        double massfrac[NSPEC];
        for (int sp = 0; sp < NSPEC; ++sp) massfrac[sp] = f(i, j, k, UFS + sp) / f(i, j, k, URHO);
        const double small_e = eos_rty2e(P.gamma, P.small_temp, massfrac);
        f(i, j, k, URHO) = P.small_dens;
        f(i, j, k, UTEMP) = P.small_temp;
        f(i, j, k, UMX) = 0.;
        f(i, j, k, UMY) = 0.;
        f(i, j, k, UMZ) = 0.;
        f(i, j, k, UEINT) = P.small_dens * small_e;
        f(i, j, k, UEDEN) = f(i, j, k, UEINT);
      } else {
        for (int q = 0; q < NVAR; ++q) f(i, j, k, q) = f(is, js, ks, q);
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) *fl.count = 0;
}

// normalize_species on the valid cells (Source/CAMR.cpp:866-908).
__global__ void __launch_bounds__(kFB) k_fab_normalize(FabSet S) {
  const FabBox& b = S.box[blockIdx.y];
  int i, j, k;
  if (!fab_region_cell(b, int64_t(blockIdx.x) * kFB + threadIdx.x, i, j, k)) return;
  if (!in_box(b, i, j, k)) return;
  double s[NVAR];
  for (int n = 0; n < NVAR; ++n) s[n] = b.f(i, j, k, n);
  normalize_species(s);
  for (int n = UFS; n < UFS + NSPEC; ++n) b.f(i, j, k, n) = s[n];
}

// normalize_species' FillBoundary (:907) then computeTemp on the ghost
// cells (:1141-1185): a ghost cell inside the (periodic) domain that some
// box's valid cells hold takes that cell's cleaned value; the others (past
// a physical boundary, or uncovered) keep theirs.  Reads valid cells only.
__global__ void __launch_bounds__(kFB) k_fab_ghost_temp(FabSet S, KParams P) {
  const FabBox& b = S.box[blockIdx.y];
  int i, j, k;
  if (!fab_region_cell(b, int64_t(blockIdx.x) * kFB + threadIdx.x, i, j, k)) return;
  if (in_box(b, i, j, k)) return;
  int src[3];
  unsigned neg;
  bool physical;
  ghost_source(S, i, j, k, src, neg, physical);
  double s[NVAR];
  int o = -1;
  if (!physical) {
    int hint = -1;
    o = find_owner(S, src[0], src[1], src[2], hint);
  }
  if (o >= 0) {
    for (int n = 0; n < NVAR; ++n) s[n] = S.box[o].f(src[0], src[1], src[2], n);
  } else {
    for (int n = 0; n < NVAR; ++n) s[n] = b.f(i, j, k, n);
  }
  compute_temp(s, P);
  for (int n = 0; n < NVAR; ++n) b.f(i, j, k, n) = s[n];
}

// computeTemp in place on every ghost cell of the fabs (within ng).
__global__ void __launch_bounds__(kFB) k_fab_ghost_temp_in_place(FabSet S, KParams P) {
  const FabBox& b = S.box[blockIdx.y];
  int i, j, k;
  if (!fab_region_cell(b, int64_t(blockIdx.x) * kFB + threadIdx.x, i, j, k)) return;
  if (in_box(b, i, j, k)) return;
  double s[NVAR];
  for (int n = 0; n < NVAR; ++n) s[n] = b.f(i, j, k, n);
  compute_temp(s, P);
  for (int n = 0; n < NVAR; ++n) b.f(i, j, k, n) = s[n];
}

// computeTemp on the valid cells (after every ghost cell has read them).
__global__ void __launch_bounds__(kFB) k_fab_valid_temp(FabSet S, KParams P) {
  const FabBox& b = S.box[blockIdx.y];
  int i, j, k;
  if (!fab_region_cell(b, int64_t(blockIdx.x) * kFB + threadIdx.x, i, j, k)) return;
  if (!in_box(b, i, j, k)) return;
  double s[NVAR];
  for (int n = 0; n < NVAR; ++n) s[n] = b.f(i, j, k, n);
  compute_temp(s, P);
  for (int n = 0; n < NVAR; ++n) b.f(i, j, k, n) = s[n];
}

// CAMR_estdt_hydro's minimum over the valid cells (Timestep.H:34-56).
__global__ void __launch_bounds__(kFB) k_fab_est_dt(FabSet S, KParams P,
                                                     unsigned long long* bits) {
  const FabBox& b = S.box[blockIdx.y];
  int i, j, k;
  double v = DBL_MAX;
  if (fab_region_cell(b, int64_t(blockIdx.x) * kFB + threadIdx.x, i, j, k) && in_box(b, i, j, k)) {
    double s[NVAR];
    for (int n = 0; n < NVAR; ++n) s[n] = b.f(i, j, k, n);
    LGeom L{};
    for (int d = 0; d < 3; ++d) L.dx[d] = S.dx[d];
    v = cell_dt(s, L, P);
  }
  block_min_dt(v, bits);
}

}  // namespace

// The library-wide error word on the current device (see scratch_address
// in noalloc.cu for why the lookup is repeated outside stream capture).
cudaError_t library_error_word(cudaStream_t st, DevError** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(st, &cap);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_err_mu);
  if (cap == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_lib_err);
    if (e != cudaSuccess) return e;
    g_err_addr[dev] = static_cast<DevError*>(p);
  } else if (!g_err_addr[dev]) {
    return cudaErrorStreamCaptureUnsupported;
  }
  *out = g_err_addr[dev];
  return cudaSuccess;
}

}  // namespace camr

using namespace camr;

namespace {

// Validates the box list and builds the device table (stream-ordered
// allocation, freed by the caller with cudaFreeAsync).
camr_status make_fabset(const camr_geom* geom, int nbox, const camr_box_fab* boxes, int ng,
                        cudaStream_t st, FabSet& S, FabBox** dev, int64_t* max_cells) {
  if (!geom || nbox <= 0 || nbox > 65535 || !boxes || ng < 0) return CAMR_ERR_INVALID;
  std::vector<FabBox> h(static_cast<size_t>(nbox));
  int64_t mx = 0;
  for (int b = 0; b < nbox; ++b) {
    const camr_box_fab& x = boxes[b];
    if (!x.fab.ptr || x.fab.ncomp < NVAR) return CAMR_ERR_INVALID;
    FabBox& o = h[size_t(b)];
    int64_t cells = 1;
    for (int d = 0; d < 3; ++d) {
      if (x.hi[d] < x.lo[d]) return CAMR_ERR_INVALID;
      if (x.lo[d] < geom->dom_lo[d] || x.hi[d] > geom->dom_hi[d]) return CAMR_ERR_INVALID;
      if (x.fab.lo[d] > x.lo[d] - ng || x.fab.hi[d] < x.hi[d] + ng) return CAMR_ERR_INVALID;
      o.lo[d] = x.lo[d];
      o.hi[d] = x.hi[d];
      o.glo[d] = x.lo[d] - ng;
      o.ghi[d] = x.hi[d] + ng;
      cells *= o.ghi[d] - o.glo[d] + 1;
    }
    o.f = make_dfab(x.fab);
    mx = cells > mx ? cells : mx;
  }
  for (int d = 0; d < 3; ++d) {
    S.dlo[d] = geom->dom_lo[d];
    S.dhi[d] = geom->dom_hi[d];
    S.periodic[d] = geom->is_periodic[d];
    S.bclo[d] = geom->bc_lo[d];
    S.bchi[d] = geom->bc_hi[d];
    S.dx[d] = geom->dx[d];
    if (!S.periodic[d] && (S.bclo[d] < 1 || S.bclo[d] > 5 || S.bchi[d] < 1 || S.bchi[d] > 5))
      return CAMR_ERR_INVALID;
  }
  S.nbox = nbox;
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(dev), sizeof(FabBox) * size_t(nbox), st);
  if (e != cudaSuccess) return CAMR_ERR_NOMEM;
  e = cudaMemcpyAsync(*dev, h.data(), sizeof(FabBox) * size_t(nbox), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) {
    cudaFreeAsync(*dev, st);
    return cuda_status_of(e);
  }
  S.box = *dev;
  *max_cells = mx;
  return CAMR_OK;
}

dim3 fab_grid(const FabSet& S, int64_t max_cells) {
  return dim3(unsigned((max_cells + kFB - 1) / kFB), unsigned(S.nbox));
}

}  // namespace

extern "C" {

camr_status camr_fill_ghosts(const camr_geom* geom, int nbox, const camr_box_fab* boxes, int ng,
                             void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  FabSet S;
  FabBox* dev = nullptr;
  int64_t mx = 0;
  camr_status cs = make_fabset(geom, nbox, boxes, ng, st, S, &dev, &mx);
  if (cs != CAMR_OK) return cs;
  if (ng > 0) {
    k_fab_fill<<<fab_grid(S, mx), kFB, 0, st>>>(S);
    count_launch();
  }
  const cudaError_t e = cudaGetLastError();
  cudaFreeAsync(dev, st);
  return cuda_status_of(e);
}

camr_status camr_clean_state_parts(const camr_geom* geom, int nbox, const camr_box_fab* boxes,
                                   int ng, const camr_hydro_params* p, int parts, void* stream) {
  if (!p || parts <= 0 || parts > 15) return CAMR_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  DevError* err = nullptr;
  cudaError_t e = library_error_word(st, &err);
  if (e != cudaSuccess) return cuda_status_of(e);
  FabSet S;
  FabBox* dev = nullptr;
  int64_t mx = 0;
  camr_status cs = make_fabset(geom, nbox, boxes, ng, st, S, &dev, &mx);
  if (cs != CAMR_OK) return cs;
  const KParams P = make_kparams(*p);
  void* fbuf = nullptr;
  if (parts & CAMR_CLEAN_VALID) {
    // the list of cells below the density floor: count, then the cells
    e = cudaMallocAsync(&fbuf, sizeof(int64_t) * (kFloorCap + 1), st);
    if (e != cudaSuccess) {
      cudaFreeAsync(dev, st);
      return CAMR_ERR_NOMEM;
    }
    FloorList fl;
    fl.count = static_cast<int*>(fbuf);
    fl.cells = static_cast<int64_t*>(fbuf) + 1;
    e = cudaMemsetAsync(fl.count, 0, sizeof(int), st);
    int64_t mv = 0;
    for (int b = 0; b < nbox; ++b) {
      const int64_t c = int64_t(boxes[b].hi[0] - boxes[b].lo[0] + 1) *
                        (boxes[b].hi[1] - boxes[b].lo[1] + 1) *
                        (boxes[b].hi[2] - boxes[b].lo[2] + 1);
      mv = c > mv ? c : mv;
    }
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(reinterpret_cast<const void*>(&k_fab_floor_walk),
                               cudaFuncAttributeMaxDynamicSharedMemorySize, int(kFloorSmem));
    if (e == cudaSuccess) {
      k_fab_floor_list<<<fab_grid(S, mv), kFB, 0, st>>>(S, P, fl);
      k_fab_floor_walk<<<1, 1024, kFloorSmem, st>>>(S, P, fl, err);
      k_fab_normalize<<<fab_grid(S, mx), kFB, 0, st>>>(S);
      count_launch(3);
    }
  }
  if (e == cudaSuccess && ng > 0 && (parts & CAMR_CLEAN_GHOSTS_FROM_OWNERS)) {
    k_fab_ghost_temp<<<fab_grid(S, mx), kFB, 0, st>>>(S, P);
    count_launch();
  }
  if (e == cudaSuccess && ng > 0 && (parts & CAMR_CLEAN_GHOSTS_TEMP)) {
    k_fab_ghost_temp_in_place<<<fab_grid(S, mx), kFB, 0, st>>>(S, P);
    count_launch();
  }
  if (e == cudaSuccess && (parts & CAMR_CLEAN_VALID_TEMP)) {
    k_fab_valid_temp<<<fab_grid(S, mx), kFB, 0, st>>>(S, P);
    count_launch();
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  if (fbuf) cudaFreeAsync(fbuf, st);
  cudaFreeAsync(dev, st);
  return cuda_status_of(e);
}

camr_status camr_clean_state(const camr_geom* geom, int nbox, const camr_box_fab* boxes, int ng,
                             const camr_hydro_params* p, void* stream) {
  return camr_clean_state_parts(geom, nbox, boxes, ng, p,
                                CAMR_CLEAN_VALID | CAMR_CLEAN_GHOSTS_FROM_OWNERS |
                                    CAMR_CLEAN_VALID_TEMP,
                                stream);
}

camr_status camr_est_dt(const camr_geom* geom, int nbox, const camr_box_fab* boxes,
                        const camr_hydro_params* p, double* dt, void* stream) {
  if (!p || !dt) return CAMR_ERR_INVALID;
  if (p->cfl <= 0.0) return CAMR_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  FabSet S;
  FabBox* dev = nullptr;
  int64_t mx = 0;
  camr_status cs = make_fabset(geom, nbox, boxes, 0, st, S, &dev, &mx);
  if (cs != CAMR_OK) return cs;
  unsigned long long* bits = nullptr;
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&bits), sizeof(*bits), st);
  if (e != cudaSuccess) {
    cudaFreeAsync(dev, st);
    return CAMR_ERR_NOMEM;
  }
  const KParams P = make_kparams(*p);
  k_reset_bits<<<1, 1, 0, st>>>(bits);
  k_fab_est_dt<<<fab_grid(S, mx), kFB, 0, st>>>(S, P, bits);
  count_launch(2);
  unsigned long long h = 0;
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, bits, sizeof(h), cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(bits, st);
  cudaFreeAsync(dev, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status_of(e);
  if (p->fixed_dt > 0.0) {
    *dt = p->fixed_dt;
    return CAMR_OK;
  }
  double dtc;
  std::memcpy(&dtc, &h, sizeof(dtc));
  // CAMR::estTimeStep (Source/CAMR.cpp:490-563)
  double estdt = p->max_dt;
  double estdt_hydro = p->max_dt / p->cfl;
  estdt_hydro = dmin(estdt_hydro, dtc);
  estdt_hydro *= p->cfl;
  if (estdt_hydro < estdt) estdt = estdt_hydro;
  *dt = estdt;
  return CAMR_OK;
}

camr_status camr_get_error(void* stream, camr_error_info* info) {
  if (!info) return CAMR_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  DevError* err = nullptr;
  cudaError_t e = library_error_word(st, &err);
  if (e != cudaSuccess) return cuda_status_of(e);
  DevError h{};
  e = cudaMemcpyAsync(&h, err, sizeof(h), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(DevError), st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status_of(e);
  info->code = h.code;
  info->i = h.i;
  info->j = h.j;
  info->k = h.k;
  return h.code ? CAMR_ERR_NUMERIC : CAMR_OK;
}

}  // extern "C"
