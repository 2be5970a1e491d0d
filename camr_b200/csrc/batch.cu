// Batched hydro over the (uneven) boxes of one level: a plan built once from
// a box work-list, run as one launch per stage for all boxes (persistent,
// grid-stride over work items), or as the plain per-box launch sequence for
// comparison.  An autotuner picks, per stage, the cells each block processes
// (chunk) and the persistent grid size, by timing the candidates on the
// plan's own boxes.
//
// The reference advances the boxes of a level one MFIter iteration at a time
// (Source/Hydro/CAMR_construct_hydro_source.cpp:71), 17-27 launches per box.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "hydro_kernels.cuh"

using namespace camr;

namespace {

// 1: every stage table carries the item of each block (one int per block);
// 0: each block binary-searches the items.
#ifndef CAMR_BATCH_BLOCKMAP
#define CAMR_BATCH_BLOCKMAP 1
#endif

constexpr int kChunks[] = {1, 2, 4};
constexpr int kNChunk = 3;

struct StageTable {
  BatchItem* items = nullptr;  // device
  int* bitem = nullptr;        // device: the item of each block (null: binary search)
  int nitems = 0;
  int64_t nblocks = 0;
};

bool stage_used(int stage, bool mol) {
  switch (stage) {
    case BS_TRACE:
    case BS_FLUX1:
    case BS_FLUX2:
    case BS_FLUX3:
      return !mol;
    case BS_MOLSLOPE:
    case BS_MOLFLUX:
      return mol;
    default:
      return true;
  }
}

}  // namespace

struct camr_batch {
  int nbox = 0;
  bool mol = false;
  bool fluxes_only = false;  // no dsdt: the caller forms the update from the fluxes
  bool has_src = false;
  KParams P;
  std::vector<BoxCtx> host_boxes;
  BoxCtx* dev_boxes = nullptr;
  double* work = nullptr;
  StageTable tab[BS_COUNT][kNChunk];
  int chunk_ix[BS_COUNT];     // chosen chunk candidate per stage
  unsigned grid[BS_COUNT];    // chosen grid (0 = one block per work unit)
  int sm_count = 0;
  bool tuned = false;
};

namespace {

camr_status fill_box(const camr_box_task& t, const camr_geom& geom, bool mol, bool need_dsdt,
                     BoxCtx& c) {
  for (int d = 0; d < 3; ++d) {
    if (t.hi[d] < t.lo[d]) return CAMR_ERR_INVALID;
    if (!t.uin.ptr || t.uin.lo[d] > t.lo[d] - NGROW || t.uin.hi[d] < t.hi[d] + NGROW)
      return CAMR_ERR_INVALID;
    if (need_dsdt && (!t.dsdt.ptr || t.dsdt.lo[d] > t.lo[d] || t.dsdt.hi[d] < t.hi[d]))
      return CAMR_ERR_INVALID;
    if (!t.flx[d].ptr) return CAMR_ERR_INVALID;
    c.g.lo[d] = t.lo[d];
    c.g.hi[d] = t.hi[d];
    c.g.dlo[d] = geom.dom_lo[d];
    c.g.dhi[d] = geom.dom_hi[d];
    c.g.bclo[d] = geom.bc_lo[d];
    c.g.bchi[d] = geom.bc_hi[d];
    c.g.dx[d] = geom.dx[d];
  }
  c.uin = make_dfab(t.uin);
  c.has_src = t.src.ptr != nullptr;
  c.src = c.has_src ? make_dfab(t.src) : c.uin;
  for (int d = 0; d < 3; ++d) c.flx[d] = make_dfab(t.flx[d]);
  c.dsdt = make_dfab(t.dsdt);
  c.mol = mol;
  c.ebflag = nullptr;
  for (int d = 0; d < 3; ++d) c.eblo[d] = c.ebn[d] = 0;
  (void)need_dsdt;
  c.w.s = make_space(t.lo, t.hi);
  return CAMR_OK;
}

cudaError_t build_tables(camr_batch* b, cudaStream_t st) {
  std::vector<BatchItem> items;
  std::vector<int> bitem;
  for (int stage = 0; stage < BS_COUNT; ++stage) {
    if (!stage_used(stage, b->mol)) continue;
    for (int ci = 0; ci < kNChunk; ++ci) {
      items.clear();
      int64_t block = 0;
      const int64_t per_block = int64_t(kBatchBlock) * kChunks[ci];
      for (int bx = 0; bx < b->nbox; ++bx) {
        Region rs[6];
        const int nr = stage_regions(stage, b->host_boxes[bx].g, rs);
        for (int s = 0; s < nr; ++s) {
          const int64_t n = rs[s].count();
          if (n == 0) continue;
          BatchItem it;
          it.block0 = block;
          it.r = rs[s];
          it.box = bx;
          it.sub = s;
          items.push_back(it);
          block += (n + per_block - 1) / per_block;
        }
      }
      StageTable& T = b->tab[stage][ci];
      T.nitems = int(items.size());
      T.nblocks = block;
      cudaError_t e = cudaMalloc(&T.items, sizeof(BatchItem) * std::max<size_t>(1, items.size()));
      if (e != cudaSuccess) return e;
      e = cudaMemcpyAsync(T.items, items.data(), sizeof(BatchItem) * items.size(),
                          cudaMemcpyHostToDevice, st);
      if (e != cudaSuccess) return e;
      if (CAMR_BATCH_BLOCKMAP && block > 0 && block < (int64_t(1) << 31)) {
        // one int per block, so that a block reads its item instead of
        // binary-searching the items' first blocks
        bitem.assign(size_t(block), 0);
        for (size_t n = 0; n < items.size(); ++n) {
          const int64_t end = (n + 1 < items.size()) ? items[n + 1].block0 : block;
          for (int64_t q = items[n].block0; q < end; ++q) bitem[size_t(q)] = int(n);
        }
        e = cudaMalloc(&T.bitem, sizeof(int) * bitem.size());
        if (e != cudaSuccess) return e;
        e = cudaMemcpyAsync(T.bitem, bitem.data(), sizeof(int) * bitem.size(),
                            cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return e;
      }
      e = cudaStreamSynchronize(st);  // `items` and `bitem` are reused for the next table
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

cudaError_t run_stage(camr_batch* b, int stage, int ci, unsigned grid, DtRef dt,
                      cudaStream_t st) {
  const StageTable& T = b->tab[stage][ci];
  return launch_batched_stage(stage, b->dev_boxes, T.items, T.nitems, T.bitem, T.nblocks,
                              kChunks[ci],
                              grid, b->P, dt, nullptr, st);
}

const int kOrderCtu[] = {BS_CTOPRIM, BS_FLATDIVU, BS_TRACE, BS_FLUX1, BS_FLUX2, BS_FLUX3,
                         BS_CONSUP};
const int kOrderMol[] = {BS_CTOPRIM, BS_FLATDIVU, BS_MOLSLOPE, BS_MOLFLUX, BS_CONSUP};

}  // namespace

namespace {

camr_status batch_create_impl(int nbox, const camr_box_task* tasks, const camr_geom* geom,
                              const camr_hydro_params* p, void* stream, bool fluxes_only,
                              camr_batch** out, const unsigned* ebflag = nullptr,
                              const int* eblo = nullptr, const int* ebn = nullptr) {
  if (nbox <= 0 || !tasks || !geom || !p || !out) return CAMR_ERR_INVALID;
  if (p->riemann_solver < 0 || p->riemann_solver > 1) return CAMR_ERR_UNSUPPORTED;
  if (!p->do_mol && p->ppm_type != 0 && p->ppm_type != 1) return CAMR_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  camr_batch* b = new (std::nothrow) camr_batch();
  if (!b) return CAMR_ERR_NOMEM;
  b->nbox = nbox;
  b->mol = p->do_mol != 0;
  b->fluxes_only = fluxes_only;
  b->P = make_kparams(*p);
  b->host_boxes.resize(nbox);
  size_t total = 0;
  std::vector<size_t> offs(nbox);
  for (int i = 0; i < nbox; ++i) {
    camr_status cs = fill_box(tasks[i], *geom, b->mol, !fluxes_only, b->host_boxes[i]);
    if (cs != CAMR_OK) {
      delete b;
      return cs;
    }
    if (ebflag) {
      BoxCtx& c = b->host_boxes[i];
      c.ebflag = ebflag;
      for (int d = 0; d < 3; ++d) {
        c.eblo[d] = eblo[d];
        c.ebn[d] = ebn[d];
        // the flags must cover the ctoprim region grow(box, 4)
        if (c.g.lo[d] - NGROW < eblo[d] || c.g.hi[d] + NGROW >= eblo[d] + ebn[d]) {
          delete b;
          return CAMR_ERR_INVALID;
        }
      }
    }
    b->has_src = b->has_src || b->host_boxes[i].has_src;
    offs[i] = total;
    size_t n = work_doubles(b->host_boxes[i].w.s, b->mol, b->host_boxes[i].has_src);
    total += (n + 31) / 32 * 32;  // 256-byte aligned slices
  }
  cudaError_t e = cudaMalloc(&b->work, total * sizeof(double));
  if (e != cudaSuccess) {
    delete b;
    return CAMR_ERR_NOMEM;
  }
  for (int i = 0; i < nbox; ++i) {
    BoxCtx& c = b->host_boxes[i];
    work_carve(c.w, b->work + offs[i], b->mol, c.has_src);
  }
  e = cudaMalloc(&b->dev_boxes, sizeof(BoxCtx) * nbox);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->dev_boxes, b->host_boxes.data(), sizeof(BoxCtx) * nbox,
                        cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = build_tables(b, st);
  int dev = 0;
  if (e == cudaSuccess) e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, dev);
  for (int s = 0; s < BS_COUNT; ++s) {
    b->chunk_ix[s] = 0;
    b->grid[s] = 0;
  }
  if (e != cudaSuccess) {
    camr_batch_destroy(b);
    return CAMR_ERR_CUDA;
  }
  *out = b;
  return CAMR_OK;
}

}  // namespace

namespace camr {

camr_status batch_create_fluxes(int nbox, const camr_box_task* tasks, const camr_geom* geom,
                                const camr_hydro_params* p, cudaStream_t st, camr_batch** out) {
  return batch_create_impl(nbox, tasks, geom, p, st, true, out);
}

const Work& batch_work(const camr_batch* b, int box) { return b->host_boxes[box].w; }

camr_status batch_create_eb(int nbox, const camr_box_task* tasks, const camr_geom* geom,
                            const camr_hydro_params* p, cudaStream_t st, const unsigned* flag,
                            const int glo[3], const int gn[3], camr_batch** out) {
  if (!flag || !glo || !gn) return CAMR_ERR_INVALID;
  return batch_create_impl(nbox, tasks, geom, p, st, false, out, flag, glo, gn);
}

}  // namespace camr

extern "C" {

camr_status camr_batch_create(int nbox, const camr_box_task* tasks, const camr_geom* geom,
                              const camr_hydro_params* p, void* stream, camr_batch** out) {
  return batch_create_impl(nbox, tasks, geom, p, stream, false, out);
}

camr_status camr_batch_destroy(camr_batch* b) {
  if (!b) return CAMR_ERR_INVALID;
  for (int s = 0; s < BS_COUNT; ++s)
    for (int c = 0; c < kNChunk; ++c) {
      if (b->tab[s][c].items) cudaFree(b->tab[s][c].items);
      if (b->tab[s][c].bitem) cudaFree(b->tab[s][c].bitem);
    }
  if (b->dev_boxes) cudaFree(b->dev_boxes);
  if (b->work) cudaFree(b->work);
  delete b;
  return CAMR_OK;
}

camr_status camr_batch_run(camr_batch* b, double dt, const double* dt_dev, int mode,
                           void* stream) {
  if (!b) return CAMR_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const DtRef dtr{dt, dt_dev};
  cudaError_t e = cudaSuccess;
  if (mode == CAMR_BATCH_PER_BOX) {
    // The plain per-box kernels, one launch sequence per box.
    for (int i = 0; i < b->nbox && e == cudaSuccess; ++i) {
      const BoxCtx& c = b->host_boxes[i];
      HydroLaunch L;
      L.g = c.g;
      L.P = b->P;
      L.uin = c.uin;
      L.src = c.src;
      L.has_src = c.has_src;
      L.mol = b->mol;
      for (int d = 0; d < 3; ++d) L.flx[d] = c.flx[d];
      L.dsdt = c.dsdt;
      L.dt = dtr;
      L.err = nullptr;
      e = b->fluxes_only ? launch_hydro_fluxes(L, c.w, st) : launch_hydro(L, c.w, st);
    }
  } else {
    const int* order = b->mol ? kOrderMol : kOrderCtu;
    const int n = (b->mol ? 5 : 7) - (b->fluxes_only ? 1 : 0);
    for (int s = 0; s < n && e == cudaSuccess; ++s) {
      const int stage = order[s];
      e = run_stage(b, stage, b->chunk_ix[stage], b->grid[stage], dtr, st);
    }
  }
  return e == cudaSuccess ? CAMR_OK : CAMR_ERR_CUDA;
}

camr_status camr_batch_autotune(camr_batch* b, double dt, void* stream) {
  if (!b) return CAMR_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const DtRef dtr{dt, nullptr};
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int* order = b->mol ? kOrderMol : kOrderCtu;
  const int n = b->mol ? 5 : 7;
  cudaError_t e = cudaSuccess;
  for (int s = 0; s < n && e == cudaSuccess; ++s) {
    const int stage = order[s];
    if (stage == BS_CONSUP) {
      // dSdt accumulates: not re-run for timing.
      b->chunk_ix[stage] = 0;
      b->grid[stage] = 0;
      break;
    }
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batched_kernel(stage), kBatchBlock, 0);
    occ = std::max(occ, 1);
    float best = 1e30f;
    int best_c = 0;
    unsigned best_g = 0;
    for (int ci = 0; ci < kNChunk && e == cudaSuccess; ++ci) {
      const unsigned grids[] = {0u, unsigned(b->sm_count * occ), unsigned(2 * b->sm_count * occ)};
      for (unsigned g : grids) {
        // one untimed launch, then the timed one
        e = run_stage(b, stage, ci, g, dtr, st);
        if (e != cudaSuccess) break;
        cudaEventRecord(e0, st);
        e = run_stage(b, stage, ci, g, dtr, st);
        cudaEventRecord(e1, st);
        if (e != cudaSuccess) break;
        e = cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) {
          best = ms;
          best_c = ci;
          best_g = g;
        }
      }
    }
    b->chunk_ix[stage] = best_c;
    b->grid[stage] = best_g;
    // leave this stage's outputs from the chosen configuration in place
    if (e == cudaSuccess) e = run_stage(b, stage, best_c, best_g, dtr, st);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->tuned = (e == cudaSuccess);
  return e == cudaSuccess ? CAMR_OK : CAMR_ERR_CUDA;
}

camr_status camr_batch_tuning(camr_batch* b, int* chunk, unsigned* grid, int n) {
  if (!b || !chunk || !grid || n < BS_COUNT) return CAMR_ERR_INVALID;
  for (int s = 0; s < BS_COUNT; ++s) {
    chunk[s] = kChunks[b->chunk_ix[s]];
    grid[s] = b->grid[s];
  }
  return CAMR_OK;
}

camr_status camr_batch_set_tuning(camr_batch* b, const int* chunk, const unsigned* grid, int n) {
  if (!b || !chunk || !grid || n < BS_COUNT) return CAMR_ERR_INVALID;
  int ix[BS_COUNT];
  for (int s = 0; s < BS_COUNT; ++s) {
    ix[s] = -1;
    for (int ci = 0; ci < kNChunk; ++ci)
      if (kChunks[ci] == chunk[s]) ix[s] = ci;
    if (ix[s] < 0) return CAMR_ERR_INVALID;
  }
  for (int s = 0; s < BS_COUNT; ++s) {
    b->chunk_ix[s] = ix[s];
    b->grid[s] = grid[s];
  }
  return CAMR_OK;
}

camr_status camr_hydro_umdrv_batched(int nbox, const camr_box_task* tasks,
                                     const camr_geom* geom, const camr_hydro_params* p,
                                     double dt, void* stream) {
  camr_batch* b = nullptr;
  camr_status cs = camr_batch_create(nbox, tasks, geom, p, stream, &b);
  if (cs != CAMR_OK) return cs;
  cs = camr_batch_run(b, dt, nullptr, CAMR_BATCH_PERSISTENT, stream);
  cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
  camr_batch_destroy(b);
  if (cs != CAMR_OK) return cs;
  return e == cudaSuccess ? CAMR_OK : CAMR_ERR_CUDA;
}

}  // extern "C"
