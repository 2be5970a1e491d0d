// Level driver on the device and the C ABI of include/camr_b200.h.
//
// One uniform level is held as padded domain arrays (the domain grown by
// NGROW ghost cells, Array4 layout).  A coarse step restates
// CAMR::CAMR_advance (Source/CAMR_advance.cpp:38-164) + post_timestep:
//   clean_state(S_old)                      k_clean_copy
//   expand_state(Sborder) = FillPatch+clean k_expand
//   hydro (construct_hydro_source)          hydro kernels on the whole domain
//   S_new = Sborder + dt*src_old + dt*dSdt,
//   clean, + dt*src_new, clean, clean,      k_update_* (one fused pass)
//   next dt: per-cell CFL min (warp shuffle, block reduce, one atomicMin on
//   order-preserving bits), then computeNewDt on one thread (k_dt_next).
// The dt lives in device memory, so the whole step is graph-capturable.
#include <cuda_runtime.h>

#include <atomic>
#include <cfloat>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "level_point.cuh"

namespace camr {

std::atomic<int64_t> g_launches{0};
void count_launch(int n) { g_launches += n; }
int64_t launches_now() { return g_launches.load(); }

static thread_local char g_last_error[256] = "";

camr_status cuda_status_of(cudaError_t e) {
  if (e == cudaSuccess) return CAMR_OK;
  std::snprintf(g_last_error, sizeof(g_last_error), "%s: %s", cudaGetErrorName(e),
                cudaGetErrorString(e));
  return CAMR_ERR_CUDA;
}
const char* last_error_text() { return g_last_error; }
void launches_sub(int64_t n) { g_launches -= n; }

}  // namespace camr

using namespace camr;

struct camr_level {
  LGeom L;
  KParams P;
  camr_hydro_params hp;
  camr_level_desc desc;
  LevelState st;
  cudaStream_t stream;
  int64_t ncell;
  int hist_cap;
  int steps_taken;
  bool graph_ready;
  cudaGraphExec_t graph;
  double* staging;     // packed (NVAR x ncell) device buffer for state input
  double* staging_out; // packed device buffer for state output
  double* fixed_dev;   // device copy of one fixed dt
  double* src_h = nullptr;  // sources_for_hydro (CTU with gravity), padded NVAR
  bool ctu_grav = false;
  FloorList floor;          // cells below the density floor of the current pass
  bool restart_est = false; // next step: CFL estimate from the state, then computeNewDt
  bool own_stream;     // the library created `stream` (caller passed NULL)
  int64_t kernels_per_step;  // launches inside one captured step
  // Host transfers run on their own streams so that the next state upload
  // and the last state download overlap the level's kernels: the upload of
  // step k+1 waits only until the unpack of step k has read `staging`, the
  // download of step k only for its own pack, and the next pack into
  // `staging_out` for the previous download.
  cudaStream_t up = nullptr, down = nullptr;
  cudaEvent_t in_free = nullptr, in_ready = nullptr, out_ready = nullptr, out_free = nullptr;
};

namespace {

camr_status cuda_status(cudaError_t e) { return camr::cuda_status_of(e); }

camr_status check_params(const camr_hydro_params* p) { return camr::check_hydro_params(p); }

}  // namespace

namespace camr {

camr_status check_hydro_params(const camr_hydro_params* p) {
  if (!p) return CAMR_ERR_INVALID;
  if (p->riemann_solver < 0 || p->riemann_solver > 1) return CAMR_ERR_UNSUPPORTED;
  if (!p->do_mol && p->ppm_type != 0 && p->ppm_type != 1) return CAMR_ERR_INVALID;
  if (p->cfl <= 0.0 || p->cfl > 1.0) return CAMR_ERR_INVALID;  // CAMR.cpp:172-174
  if (p->do_mol && p->cfl > 0.3 && p->fixed_dt <= 0.0) return CAMR_ERR_INVALID;  // :175-177
  return CAMR_OK;
}

}  // namespace camr

extern "C" {

void camr_default_params(camr_hydro_params* p) {
  std::memset(p, 0, sizeof(*p));
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
  p->riemann_solver = 0;
  p->eb_weights_type = 2;
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
  p->eos_gamma = 1.4;      // Source/EOS/GammaLaw/EOS.H:16
  p->smallu = 1.e-12;      // Source/Utils/CAMR_Constants.H:9
  p->small_num = 1.e-8;    // Source/Utils/CAMR_Constants.H:10
}

const char* camr_version(void) { return "camr_b200 0.1 (sm_100a, FP64)"; }

int64_t camr_launch_count(void) { return g_launches.load(); }

}  // extern "C"

namespace {

// The per-box hydro behind camr_hydro_umdrv and camr_hydro_umdrv_full: q
// (with qaux and the primitive sources src_q) either from ctoprim /
// srctoprim of uin and src, or the caller's; area/vol either Cartesian from
// dx or the caller's.
camr_status umdrv_common(const int bx_lo[3], const int bx_hi[3], const camr_geom* geom,
                         const camr_fab* uin, const camr_fab* src, const camr_fab* q,
                         const camr_fab* qaux, const camr_fab* src_q, camr_fab* dsdt,
                         camr_fab* flx0, camr_fab* flx1, camr_fab* flx2,
                         const camr_fab* const* area, const camr_fab* vol,
                         const camr_hydro_params* p, double dt, void* stream) {
  if (!bx_lo || !bx_hi || !geom || !uin || !dsdt || !flx0 || !flx1 || !flx2 || !uin->ptr ||
      !dsdt->ptr || !flx0->ptr || !flx1->ptr || !flx2->ptr)
    return CAMR_ERR_INVALID;
  camr_status cs = check_params(p);
  if (cs != CAMR_OK) return cs;
  auto covers = [&](const camr_fab* f, int grow, int hi_extra_dir) {
    for (int d = 0; d < 3; ++d) {
      const int hx = (d == hi_extra_dir) ? 1 : 0;
      if (f->lo[d] > bx_lo[d] - grow || f->hi[d] < bx_hi[d] + grow + hx) return false;
    }
    return true;
  };
  for (int d = 0; d < 3; ++d)
    if (bx_hi[d] < bx_lo[d]) return CAMR_ERR_INVALID;
  // uin must cover grow(bx, 4)
  if (!covers(uin, NGROW, -1) || !covers(dsdt, 0, -1)) return CAMR_ERR_INVALID;
  if (src && src->ptr && !covers(src, NGROW, -1)) return CAMR_ERR_INVALID;
  if (uin->ncomp < NVAR || dsdt->ncomp < NVAR) return CAMR_ERR_INVALID;
  const bool ext_q = q != nullptr;
  if (ext_q) {
    if (!q->ptr || !qaux || !qaux->ptr || q->ncomp < QVAR || qaux->ncomp < NQAUX ||
        !covers(q, NGROW, -1) || !covers(qaux, NGROW, -1))
      return CAMR_ERR_INVALID;
    if (src_q && (!src_q->ptr || src_q->ncomp < QVAR || !covers(src_q, NGROW, -1)))
      return CAMR_ERR_INVALID;
  }
  const bool met = area != nullptr;
  if (met) {
    for (int d = 0; d < 3; ++d)
      if (!area[d] || !area[d]->ptr || !covers(area[d], 0, d)) return CAMR_ERR_INVALID;
    if (!vol || !vol->ptr || !covers(vol, 0, -1)) return CAMR_ERR_INVALID;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  HydroLaunch Lh;
  for (int d = 0; d < 3; ++d) {
    Lh.g.lo[d] = bx_lo[d];
    Lh.g.hi[d] = bx_hi[d];
    Lh.g.dlo[d] = geom->dom_lo[d];
    Lh.g.dhi[d] = geom->dom_hi[d];
    Lh.g.bclo[d] = geom->bc_lo[d];
    Lh.g.bchi[d] = geom->bc_hi[d];
    Lh.g.dx[d] = geom->dx[d];
  }
  Lh.P = make_kparams(*p);
  Lh.uin = make_dfab(*uin);
  Lh.has_src = src && src->ptr;
  Lh.src = Lh.has_src ? make_dfab(*src) : Lh.uin;
  if (ext_q) {
    Lh.ext_q = true;
    Lh.qin = make_dfab(*q);
    Lh.qauxin = make_dfab(*qaux);
    Lh.ext_srcq = src_q != nullptr;
    Lh.srcqin = Lh.ext_srcq ? make_dfab(*src_q) : Lh.qin;
    Lh.has_src = Lh.ext_srcq;  // the srcq array holds the caller's sources
  }
  if (met) {
    for (int d = 0; d < 3; ++d) Lh.M.a[d] = make_dfab(*area[d]);
    Lh.M.vol = make_dfab(*vol);
    Lh.M.on = 1;
  }
  Lh.mol = p->do_mol != 0;
  Lh.flx[0] = make_dfab(*flx0);
  Lh.flx[1] = make_dfab(*flx1);
  Lh.flx[2] = make_dfab(*flx2);
  Lh.dsdt = make_dfab(*dsdt);
  Lh.dt = DtRef{dt, nullptr};
  // ctoprim's checks (Hydro_ctoprim.H:56,68) report into the library's
  // error word (camr_get_error) where the reference asserts
  cudaError_t ee = library_error_word(st, &Lh.err);
  if (ee != cudaSuccess) return cuda_status(ee);
  Work w;
  w.s = make_space(bx_lo, bx_hi);
  const size_t bytes = work_doubles(w.s, Lh.mol, Lh.has_src) * sizeof(double);
  double* base = nullptr;
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&base), bytes, st);
  if (e != cudaSuccess) return CAMR_ERR_NOMEM;
  work_carve(w, base, Lh.mol, Lh.has_src);
  e = launch_hydro(Lh, w, st);
  cudaError_t e2 = cudaFreeAsync(base, st);
  if (e != cudaSuccess) return cuda_status(e);
  return cuda_status(e2);
}

}  // namespace

extern "C" {

camr_status camr_hydro_umdrv(const int bx_lo[3], const int bx_hi[3], const camr_geom* geom,
                             const camr_fab* uin, const camr_fab* src, camr_fab* dsdt,
                             camr_fab* flx0, camr_fab* flx1, camr_fab* flx2,
                             const camr_hydro_params* p, double dt, void* stream) {
  return umdrv_common(bx_lo, bx_hi, geom, uin, src, nullptr, nullptr, nullptr, dsdt, flx0, flx1,
                      flx2, nullptr, nullptr, p, dt, stream);
}

camr_status camr_hydro_umdrv_full(const int bx_lo[3], const int bx_hi[3], const camr_geom* geom,
                                  const camr_fab* uin, const camr_fab* q, const camr_fab* qaux,
                                  const camr_fab* src_q, camr_fab* dsdt, camr_fab* flx0,
                                  camr_fab* flx1, camr_fab* flx2, const camr_fab* area0,
                                  const camr_fab* area1, const camr_fab* area2,
                                  const camr_fab* vol, const camr_hydro_params* p, double dt,
                                  void* stream) {
  if (!q || !qaux) return CAMR_ERR_INVALID;
  const bool met = area0 || area1 || area2 || vol;
  const camr_fab* area[3] = {area0, area1, area2};
  return umdrv_common(bx_lo, bx_hi, geom, uin, nullptr, q, qaux, src_q, dsdt, flx0, flx1, flx2,
                      met ? area : nullptr, vol, p, dt, stream);
}

camr_status camr_level_create(const camr_level_desc* desc, const camr_hydro_params* p,
                              void* stream, camr_level** out) {
  if (!desc || !out) return CAMR_ERR_INVALID;
  camr_status cs = check_params(p);
  if (cs != CAMR_OK) return cs;
  if (floor_prepare() != cudaSuccess) return CAMR_ERR_CUDA;
  camr_level* lev = new (std::nothrow) camr_level();
  if (!lev) return CAMR_ERR_NOMEM;
  lev->hp = *p;
  lev->P = make_kparams(*p);
  lev->desc = *desc;
  lev->stream = static_cast<cudaStream_t>(stream);
  if (!lev->stream) {
    // The legacy default stream cannot be captured into a graph: give the
    // level its own stream (camr_level_stream returns it).
    if (cudaStreamCreateWithFlags(&lev->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete lev;
      return CAMR_ERR_CUDA;
    }
    lev->own_stream = true;
  }
  LGeom& L = lev->L;
  const camr_geom& g = desc->geom;
  for (int d = 0; d < 3; ++d) {
    if (g.dom_hi[d] < g.dom_lo[d]) { delete lev; return CAMR_ERR_INVALID; }
    if (!g.is_periodic[d] && (g.bc_lo[d] == CAMR_BC_INTERIOR || g.bc_hi[d] == CAMR_BC_INTERIOR)) {
      delete lev;
      return CAMR_ERR_INVALID;  // CAMR.cpp:147-156
    }
    L.dlo[d] = g.dom_lo[d];
    L.dhi[d] = g.dom_hi[d];
    L.plo[d] = g.dom_lo[d] - NGROW;
    // the hydro Space of the domain box (one extra high layer for faces)
    L.pn[d] = g.dom_hi[d] - g.dom_lo[d] + 1 + 2 * NGROW;
    L.periodic[d] = g.is_periodic[d];
    L.bclo[d] = g.bc_lo[d];
    L.bchi[d] = g.bc_hi[d];
    L.dx[d] = g.dx[d];
    const int n = g.dom_hi[d] - g.dom_lo[d] + 1;
    L.boxsz[d] = desc->max_grid_size[d] > 0 ? desc->max_grid_size[d] : n;
  }
  // State arrays share the hydro Space's layout so that Sborder can be the
  // hydro input directly.
  const Space sp = make_space(L.dlo, L.dhi);
  L.sy = sp.sy;
  L.sz = sp.sz;
  L.sn = sp.sn;
  lgeom_finish(L);
  lev->ncell = int64_t(L.dhi[0] - L.dlo[0] + 1) * (L.dhi[1] - L.dlo[1] + 1) *
               (L.dhi[2] - L.dlo[2] + 1);
  lev->hist_cap = 1 << 16;
  LevelState& S = lev->st;
  const bool mol = p->do_mol != 0;
  // A CTU step with gravity feeds the old-time source into the hydro
  // (hydro_srctoprim); with const_grav = 0 every source term is +0, which
  // the kernels reproduce without a source array.
  lev->ctu_grav = !mol && p->add_grav_src && p->const_grav != 0.0;
  const size_t state_bytes = size_t(sp.sn) * NVAR * sizeof(double);
  const size_t work_bytes = work_doubles(sp, mol, lev->ctu_grav) * sizeof(double);
  cudaError_t e = cudaSuccess;
  // Zero-fill on the level's own stream: a non-blocking stream does not
  // order against the legacy default stream, so a plain cudaMemset could
  // land after the first upload into the same buffer.
  auto alloc = [&](void** ptr, size_t b) {
    if (e == cudaSuccess) e = cudaMalloc(ptr, b);
    if (e == cudaSuccess) e = cudaMemsetAsync(*ptr, 0, b, lev->stream);
  };
  alloc(reinterpret_cast<void**>(&S.S), state_bytes);
  alloc(reinterpret_cast<void**>(&S.S_old), state_bytes);
  alloc(reinterpret_cast<void**>(&S.B), state_bytes);
  if (mol) alloc(reinterpret_cast<void**>(&S.B2), state_bytes);
  for (int d = 0; d < 3; ++d) alloc(reinterpret_cast<void**>(&S.flx[d]), state_bytes);
  alloc(reinterpret_cast<void**>(&S.work), work_bytes);
  if (lev->ctu_grav) alloc(reinterpret_cast<void**>(&lev->src_h), state_bytes);
  alloc(reinterpret_cast<void**>(&S.dt_cur), sizeof(double));
  alloc(reinterpret_cast<void**>(&S.dt_hist), sizeof(double) * lev->hist_cap);
  alloc(reinterpret_cast<void**>(&S.dtmin_bits), sizeof(unsigned long long));
  alloc(reinterpret_cast<void**>(&S.nstep), sizeof(int));
  alloc(reinterpret_cast<void**>(&S.err), sizeof(DevError));
  alloc(reinterpret_cast<void**>(&lev->staging), size_t(lev->ncell) * NVAR * sizeof(double));
  alloc(reinterpret_cast<void**>(&lev->staging_out), size_t(lev->ncell) * NVAR * sizeof(double));
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&lev->up, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&lev->down, cudaStreamNonBlocking);
  for (cudaEvent_t* ev : {&lev->in_free, &lev->in_ready, &lev->out_ready, &lev->out_free})
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
  alloc(reinterpret_cast<void**>(&lev->fixed_dev), sizeof(double));
  alloc(reinterpret_cast<void**>(&lev->floor.count), sizeof(int));
  alloc(reinterpret_cast<void**>(&lev->floor.cells), sizeof(int64_t) * kFloorCap);
  alloc(reinterpret_cast<void**>(&lev->floor.enforced), sizeof(double) * NVAR * kFloorCap);
  alloc(reinterpret_cast<void**>(&lev->floor.total), sizeof(unsigned long long));
  if (e != cudaSuccess) {
    camr_level_destroy(lev);
    return CAMR_ERR_NOMEM;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(lev->stream);
  if (e != cudaSuccess) {
    camr_level_destroy(lev);
    return cuda_status(e);
  }
  S.w.s = sp;
  work_carve(S.w, S.work, mol, lev->ctu_grav);
  *out = lev;
  return CAMR_OK;
}

camr_status camr_level_destroy(camr_level* lev) {
  if (!lev) return CAMR_ERR_INVALID;
  LevelState& S = lev->st;
  if (lev->graph_ready) cudaGraphExecDestroy(lev->graph);
  if (lev->up) cudaStreamSynchronize(lev->up);
  if (lev->down) cudaStreamSynchronize(lev->down);
  void* ptrs[] = {S.S,        S.S_old,  S.B,        S.B2,         S.flx[0],
                  S.flx[1],   S.flx[2], S.work,     S.dt_cur,     S.dt_hist,
                  S.dtmin_bits, S.nstep, S.err,     lev->staging, lev->staging_out,
                  lev->fixed_dev, lev->src_h, lev->floor.count, lev->floor.cells,
                  lev->floor.enforced, lev->floor.total};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (cudaEvent_t ev : {lev->in_free, lev->in_ready, lev->out_ready, lev->out_free})
    if (ev) cudaEventDestroy(ev);
  if (lev->up) cudaStreamDestroy(lev->up);
  if (lev->down) cudaStreamDestroy(lev->down);
  if (lev->own_stream) cudaStreamDestroy(lev->stream);
  delete lev;
  return CAMR_OK;
}

camr_status camr_level_set_state(camr_level* lev, const double* state, int host) {
  if (!lev || !state) return CAMR_ERR_INVALID;
  const size_t bytes = size_t(lev->ncell) * NVAR * sizeof(double);
  cudaError_t e;
  if (host) {
    // upload on the copy stream once the previous unpack has read staging
    e = cudaStreamWaitEvent(lev->up, lev->in_free, 0);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(lev->staging, state, bytes, cudaMemcpyHostToDevice, lev->up);
    if (e == cudaSuccess) e = cudaEventRecord(lev->in_ready, lev->up);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(lev->stream, lev->in_ready, 0);
  } else {
    e = cudaMemcpyAsync(lev->staging, state, bytes, cudaMemcpyDeviceToDevice, lev->stream);
  }
  if (e != cudaSuccess) return cuda_status(e);
  k_pack<<<grid_of(lev->ncell), kBlk, 0, lev->stream>>>(lev->L, lev->st.S, lev->staging, 0);
  count_launch();
  e = cudaEventRecord(lev->in_free, lev->stream);
  lev->steps_taken = 0;
  if (e != cudaSuccess) return cuda_status(e);
  return cuda_status(cudaGetLastError());
}

// Pack the state and start its copy to `state`; host copies run on the
// download stream and complete by the next camr_level_sync (or any call
// that synchronises the level).
static camr_status get_state_issue(camr_level* lev, double* state, int host) {
  cudaError_t e = cudaStreamWaitEvent(lev->stream, lev->out_free, 0);
  if (e != cudaSuccess) return cuda_status(e);
  k_pack<<<grid_of(lev->ncell), kBlk, 0, lev->stream>>>(lev->L, lev->st.S, lev->staging_out, 1);
  count_launch();
  const size_t bytes = size_t(lev->ncell) * NVAR * sizeof(double);
  if (host) {
    e = cudaEventRecord(lev->out_ready, lev->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(lev->down, lev->out_ready, 0);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(state, lev->staging_out, bytes, cudaMemcpyDeviceToHost, lev->down);
    if (e == cudaSuccess) e = cudaEventRecord(lev->out_free, lev->down);
  } else {
    e = cudaMemcpyAsync(state, lev->staging_out, bytes, cudaMemcpyDeviceToDevice, lev->stream);
  }
  if (e != cudaSuccess) return cuda_status(e);
  return cuda_status(cudaGetLastError());
}

camr_status camr_level_get_state(camr_level* lev, double* state, int host) {
  if (!lev || !state) return CAMR_ERR_INVALID;
  camr_status cs = get_state_issue(lev, state, host);
  if (cs != CAMR_OK) return cs;
  return cuda_status(cudaStreamSynchronize(host ? lev->down : lev->stream));
}

camr_status camr_level_get_state_async(camr_level* lev, double* state, int host) {
  if (!lev || !state) return CAMR_ERR_INVALID;
  return get_state_issue(lev, state, host);
}

camr_status camr_level_sync(camr_level* lev) {
  if (!lev) return CAMR_ERR_INVALID;
  cudaError_t e = cudaStreamSynchronize(lev->up);
  if (e == cudaSuccess) e = cudaStreamSynchronize(lev->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(lev->down);
  return cuda_status(e);
}

camr_status camr_level_init_finalize(camr_level* lev) {
  if (!lev) return CAMR_ERR_INVALID;
  k_init_finalize<<<grid_of(lev->ncell), kBlk, 0, lev->stream>>>(lev->L, lev->P, lev->st.S);
  count_launch();
  return cuda_status(cudaGetLastError());
}

static cudaError_t issue_step(camr_level* lev, bool first, const double* fixed_dev,
                              StageTimer* tm = nullptr, bool est = false) {
  LevelState& S = lev->st;
  const LGeom& L = lev->L;
  cudaStream_t st = lev->stream;
  const unsigned gv = grid_of(lev->ncell);
  const int64_t npad = int64_t(L.pn[0]) * L.pn[1] * L.pn[2];
  DtCtl c{lev->hp.cfl, lev->hp.max_dt, lev->hp.fixed_dt, lev->hp.initial_dt,
          lev->hp.init_shrink, lev->hp.change_max};
  auto mark = [&](const char* what) {
    if (tm) tm->mark(st, what);
  };
  if (first || est) {
    mark("est_dt");
    k_reset_bits<<<1, 1, 0, st>>>(S.dtmin_bits);
    k_est_dt<<<gv, kBlk, 0, st>>>(L, lev->P, S.S, S.dtmin_bits);
    count_launch(2);
  }
  // dt of this step (computeInitialDt / computeNewDt) from the CFL min of
  // the current state.
  mark("dt_next");
  k_dt_next<<<1, 1, 0, st>>>(c, first ? 1 : 0, fixed_dev, S.dtmin_bits, S.dt_cur, S.dt_hist,
                             S.nstep, lev->hist_cap);
  // Each cleaning pass lists the cells below the density floor and a
  // one-block fixup resets them in the reference's order (a no-op launch
  // when the list is empty).
  const FloorList& fl = lev->floor;
  auto fixup = [&](int mode, FloorArgs a) {
    switch (mode) {
      case FLOOR_CLEAN: k_floor_fixup<FLOOR_CLEAN><<<1, 1024, kFloorSmem, st>>>(L, lev->P, fl, a, S.err); break;
      case FLOOR_EXPAND: k_floor_fixup<FLOOR_EXPAND><<<1, 1024, kFloorSmem, st>>>(L, lev->P, fl, a, S.err); break;
      case FLOOR_CTU: k_floor_fixup<FLOOR_CTU><<<1, 1024, kFloorSmem, st>>>(L, lev->P, fl, a, S.err); break;
      default: k_floor_fixup<FLOOR_MOL2><<<1, 1024, kFloorSmem, st>>>(L, lev->P, fl, a, S.err); break;
    }
    count_launch();
  };
  FloorArgs fa{};
  mark("clean_copy");
  k_clean_copy<<<gv, kBlk, 0, st>>>(L, lev->P, S.S, S.S_old, S.err, fl);
  fa.in = S.S;
  fa.out = S.S_old;
  fixup(FLOOR_CLEAN, fa);
  mark("expand");
  k_expand<<<grid_of(npad), kBlk, 0, st>>>(L, lev->P, S.S_old, S.B, S.err, fl);
  fa.in = S.S_old;
  fa.out = S.B;
  fixup(FLOOR_EXPAND, fa);
  count_launch(3);
  HydroLaunch H;
  for (int d = 0; d < 3; ++d) {
    H.g.lo[d] = L.dlo[d];
    H.g.hi[d] = L.dhi[d];
    H.g.dlo[d] = L.dlo[d];
    H.g.dhi[d] = L.dhi[d];
    H.g.bclo[d] = L.bclo[d];
    H.g.bchi[d] = L.bchi[d];
    H.g.dx[d] = L.dx[d];
  }
  H.P = lev->P;
  H.has_src = false;
  H.mol = lev->hp.do_mol != 0;
  H.dt = DtRef{0.0, S.dt_cur};
  H.err = reinterpret_cast<DevError*>(S.err);
  H.timer = tm;
  auto sdfab = [&](double* p) {
    DFab f;
    f.p = p;
    for (int d = 0; d < 3; ++d) f.lo[d] = L.plo[d];
    f.sy = L.sy;
    f.sz = L.sz;
    f.sn = L.sn;
    return f;
  };
  for (int d = 0; d < 3; ++d) H.flx[d] = sdfab(S.flx[d]);
  H.dsdt = sdfab(nullptr);
  FluxPtrs fp;
  for (int d = 0; d < 3; ++d) {
    fp.f[d] = S.flx[d];
    fp.q[d] = S.w.qf[d];
  }
  const Space& sp = S.w.s;
  H.uin = sdfab(S.B);
  H.src = H.uin;
  if (lev->ctu_grav) {
    mark("src_hydro");
    k_src_hydro<<<grid_of(npad), kBlk, 0, st>>>(L, lev->P, S.S_old, lev->src_h);
    count_launch();
    H.has_src = true;
    H.src = sdfab(lev->src_h);
  }
  cudaError_t e = launch_hydro_fluxes(H, S.w, st);
  if (e != cudaSuccess) return e;
  if (!H.mol) {
    mark("update");
    k_update_ctu<<<gv, kBlk, 0, st>>>(L, sp, lev->P, S.dt_cur, S.B, S.S_old, fp, S.S,
                                      S.dtmin_bits, S.err, 1, fl);
    count_launch();
    FloorArgs fu{nullptr, S.S, S.B, S.S_old, fp, sp, S.dt_cur, S.dtmin_bits, 1};
    fixup(FLOOR_CTU, fu);
  } else {
    mark("update_mol1");
    k_update_mol1<<<gv, kBlk, 0, st>>>(L, sp, lev->P, S.dt_cur, S.B, S.S_old, fp, S.S);
    mark("expand2");
    k_expand<<<grid_of(npad), kBlk, 0, st>>>(L, lev->P, S.S, S.B2, S.err, fl);
    count_launch(2);
    fa.in = S.S;
    fa.out = S.B2;
    fixup(FLOOR_EXPAND, fa);
    H.uin = sdfab(S.B2);
    H.src = H.uin;
    e = launch_hydro_fluxes(H, S.w, st);
    if (e != cudaSuccess) return e;
    mark("update_mol2");
    k_update_mol2<<<gv, kBlk, 0, st>>>(L, sp, lev->P, S.dt_cur, S.B2, S.S_old, fp, S.S,
                                       S.dtmin_bits, S.err, 1, fl);
    count_launch();
    FloorArgs fu{nullptr, S.S, S.B2, S.S_old, fp, sp, S.dt_cur, S.dtmin_bits, 1};
    fixup(FLOOR_MOL2, fu);
  }
  mark("end");
  return cudaGetLastError();
}

camr_status camr_level_advance(camr_level* lev, int nsteps, const double* fixed_dts) {
  if (!lev || nsteps < 0) return CAMR_ERR_INVALID;
  for (int s = 0; s < nsteps; ++s) {
    const bool first = lev->steps_taken == 0;
    const double* fixed_dev = nullptr;
    if (fixed_dts) {
      cudaError_t e = cudaMemcpyAsync(lev->fixed_dev, &fixed_dts[s], sizeof(double),
                                      cudaMemcpyHostToDevice, lev->stream);
      if (e != cudaSuccess) return CAMR_ERR_CUDA;
      // the pageable source must outlive the copy
      e = cudaStreamSynchronize(lev->stream);
      if (e != cudaSuccess) return CAMR_ERR_CUDA;
      fixed_dev = lev->fixed_dev;
    }
    cudaError_t e;
    if (lev->restart_est) {
      // the first step after a restart: estTimeStep on the restored state,
      // then computeNewDt against the checkpoint's dt (uncaptured)
      lev->restart_est = false;
      e = issue_step(lev, false, fixed_dev, nullptr, true);
    } else if (!first && !fixed_dts && lev->desc.use_graph) {
      if (!lev->graph_ready) {
        cudaGraph_t g;
        e = cudaStreamBeginCapture(lev->stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return cuda_status(e);
        const int64_t before = g_launches.load();
        cudaError_t e1 = issue_step(lev, false, nullptr);
        // issuing during capture counted the kernels once; replays add them
        lev->kernels_per_step = g_launches.load() - before;
        g_launches -= lev->kernels_per_step;
        e = cudaStreamEndCapture(lev->stream, &g);
        if (e1 != cudaSuccess) return cuda_status(e1);
        if (e != cudaSuccess) return cuda_status(e);
        e = cudaGraphInstantiate(&lev->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_status(e);
        lev->graph_ready = true;
      }
      e = cudaGraphLaunch(lev->graph, lev->stream);
      count_launch(int(lev->kernels_per_step));
    } else {
      e = issue_step(lev, first, fixed_dev);
    }
    if (e != cudaSuccess) return cuda_status(e);
    lev->steps_taken++;
  }
  return CAMR_OK;
}

camr_status camr_level_last_dt(camr_level* lev, double* dt) {
  if (!lev || !dt) return CAMR_ERR_INVALID;
  cudaError_t e = cudaMemcpyAsync(dt, lev->st.dt_cur, sizeof(double), cudaMemcpyDeviceToHost,
                                  lev->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(lev->stream);
  return cuda_status(e);
}

camr_status camr_level_est_dt(camr_level* lev, double* dt) {
  if (!lev || !dt) return CAMR_ERR_INVALID;
  LevelState& S = lev->st;
  unsigned long long* tmp = nullptr;
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&tmp), sizeof(*tmp), lev->stream);
  if (e != cudaSuccess) return CAMR_ERR_NOMEM;
  k_reset_bits<<<1, 1, 0, lev->stream>>>(tmp);
  k_est_dt<<<grid_of(lev->ncell), kBlk, 0, lev->stream>>>(lev->L, lev->P, S.S, tmp);
  count_launch(2);
  unsigned long long bits = 0;
  e = cudaMemcpyAsync(&bits, tmp, sizeof(bits), cudaMemcpyDeviceToHost, lev->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(lev->stream);
  cudaFreeAsync(tmp, lev->stream);
  if (e != cudaSuccess) return CAMR_ERR_CUDA;
  double dtc;
  std::memcpy(&dtc, &bits, sizeof(dtc));
  const camr_hydro_params& p = lev->hp;
  if (p.fixed_dt > 0.0) {
    *dt = p.fixed_dt;
    return CAMR_OK;
  }
  double estdt = p.max_dt;
  double estdt_hydro = p.max_dt / p.cfl;
  estdt_hydro = dmin(estdt_hydro, dtc);
  estdt_hydro *= p.cfl;
  if (estdt_hydro < estdt) estdt = estdt_hydro;
  *dt = estdt;
  return CAMR_OK;
}

camr_status camr_level_profile_step(camr_level* lev, float* stage_ms, const char** names,
                                    int max_stages, int* nstages) {
  if (!lev || !stage_ms || !nstages || lev->steps_taken == 0) return CAMR_ERR_INVALID;
  StageTimer tm;
  for (int i = 0; i < StageTimer::kMax; ++i) {
    if (cudaEventCreate(&tm.ev[i]) != cudaSuccess) return CAMR_ERR_CUDA;
  }
  cudaError_t e = issue_step(lev, false, nullptr, &tm);
  if (e == cudaSuccess) e = cudaEventSynchronize(tm.ev[tm.n - 1]);
  int ns = 0;
  for (int i = 0; i + 1 < tm.n && ns < max_stages; ++i, ++ns) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, tm.ev[i], tm.ev[i + 1]);
    stage_ms[ns] = ms;
    if (names) names[ns] = tm.name[i];
  }
  *nstages = ns;
  for (int i = 0; i < StageTimer::kMax; ++i) cudaEventDestroy(tm.ev[i]);
  lev->steps_taken++;
  return cuda_status(e);
}

int64_t camr_level_kernels_per_step(camr_level* lev) {
  return lev ? lev->kernels_per_step : 0;
}

camr_status camr_level_stream(camr_level* lev, void** stream) {
  if (!lev || !stream) return CAMR_ERR_INVALID;
  *stream = static_cast<void*>(lev->stream);
  return CAMR_OK;
}

const char* camr_last_error_string(void) { return last_error_text(); }

camr_status camr_level_state_fab(camr_level* lev, camr_fab* fab) {
  if (!lev || !fab) return CAMR_ERR_INVALID;
  fab->ptr = lev->st.S;
  for (int d = 0; d < 3; ++d) {
    fab->lo[d] = lev->L.plo[d];
    fab->hi[d] = lev->L.dhi[d] + NGROW;
  }
  fab->jstride = lev->L.sy;
  fab->kstride = lev->L.sz;
  fab->nstride = lev->L.sn;
  fab->ncomp = NVAR;
  return CAMR_OK;
}

camr_status camr_level_restart(camr_level* lev, double dt_prev, int steps_done) {
  if (!lev || !(dt_prev > 0.0) || steps_done < 1) return CAMR_ERR_INVALID;
  cudaError_t e = cudaMemcpyAsync(lev->st.dt_cur, &dt_prev, sizeof(double),
                                  cudaMemcpyHostToDevice, lev->stream);
  // the pageable source must outlive the copy
  if (e == cudaSuccess) e = cudaStreamSynchronize(lev->stream);
  if (e != cudaSuccess) return cuda_status(e);
  lev->steps_taken = steps_done;
  lev->restart_est = true;
  return CAMR_OK;
}

camr_status camr_level_floor_resets(camr_level* lev, int64_t* cells) {
  if (!lev || !cells) return CAMR_ERR_INVALID;
  unsigned long long h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, lev->floor.total, sizeof(h), cudaMemcpyDeviceToHost,
                                  lev->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(lev->stream);
  if (e != cudaSuccess) return cuda_status(e);
  *cells = int64_t(h);
  return CAMR_OK;
}

camr_status camr_level_get_error(camr_level* lev, camr_error_info* info) {
  if (!lev || !info) return CAMR_ERR_INVALID;
  DevError h;
  cudaError_t e = cudaMemcpyAsync(&h, lev->st.err, sizeof(h), cudaMemcpyDeviceToHost, lev->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(lev->st.err, 0, sizeof(DevError), lev->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(lev->stream);
  if (e != cudaSuccess) return CAMR_ERR_CUDA;
  info->code = h.code;
  info->i = h.i;
  info->j = h.j;
  info->k = h.k;
  return h.code ? CAMR_ERR_NUMERIC : CAMR_OK;
}

}  // extern "C"
