// camr_hydro_umdrv_noalloc: the per-box hydro with its scratch in a fixed,
// statically allocated device array instead of a stream-ordered allocation.
//
// Who needs this: callers that must not allocate device memory while they
// run the hydro -- code inside a custom memory-pool or arena that owns all
// device memory (AMReX-style arenas), real-time loops that forbid
// allocator calls after start-up, and integrations (other runtimes, signal
// handlers, plugin hosts) where calling cudaMalloc/cudaMallocAsync is not
// permitted or would fight another allocator.
//
// Limits: the scratch holds CAMR_NOALLOC_SCRATCH_BYTES (64 MiB), enough for
// a cubic CTU box of up to 28^3 cells or a MOL box of up to 49^3 without a
// source fab (with one, CTU boxes up to 27^3); larger boxes are rejected
// with CAMR_ERR_INVALID (use camr_hydro_umdrv for them).
// The array lives in every GPU that loads this library until the process
// exits.  All calls share the one array: calls that overlap on the GPU (two
// streams, two host threads) race on it and must be serialised by the caller.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "hydro_kernels.cuh"

namespace {

constexpr size_t kScratchBytes = CAMR_NOALLOC_SCRATCH_BYTES;

// The scratch itself.  Host code may not use its name as an address (that
// is a host-side stand-in); the device address comes from
// cudaGetSymbolAddress, looked up once per device.
static __device__ __align__(256) double g_noalloc_scratch[kScratchBytes / sizeof(double)];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {};
thread_local char g_msg[200] = "";

// The scratch's device address on the current device.  Outside stream
// capture it is looked up again on every call (a cheap table lookup once
// the module is loaded), so a device reset, which reloads the module at a
// new address, never leaves a stale pointer behind.  While `st` is being
// captured the address cached by the last uncaptured call on this device
// is used: the first call on a device must come before any capture.
cudaError_t scratch_address(cudaStream_t st, void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(st, &cap);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_mu);
  if (cap == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_addr[dev] = p;
  } else if (!g_addr[dev]) {
    return cudaErrorStreamCaptureUnsupported;
  }
  *out = g_addr[dev];
  return cudaSuccess;
}

camr_status reject(camr_status s, const char* why) {
  std::snprintf(g_msg, sizeof(g_msg), "%s", why);
  return s;
}

}  // namespace

extern "C" const char* camr_noalloc_last_error(void) { return g_msg; }

extern "C" camr_status camr_hydro_umdrv_noalloc(const int bx_lo[3], const int bx_hi[3],
                                                const camr_geom* geom, const camr_fab* uin,
                                                const camr_fab* src, camr_fab* dsdt,
                                                camr_fab* flx0, camr_fab* flx1, camr_fab* flx2,
                                                const camr_hydro_params* p, double dt,
                                                void* stream) {
  using namespace camr;
  g_msg[0] = '\0';
  if (!bx_lo || !bx_hi || !geom || !uin || !dsdt || !flx0 || !flx1 || !flx2 || !p ||
      !uin->ptr || !dsdt->ptr || !flx0->ptr || !flx1->ptr || !flx2->ptr)
    return reject(CAMR_ERR_INVALID, "a required pointer is NULL");
  // the same parameter checks as camr_hydro_umdrv
  const camr_status cs = check_hydro_params(p);
  if (cs != CAMR_OK) return reject(cs, "parameters rejected (as camr_hydro_umdrv rejects them)");
  for (int d = 0; d < 3; ++d) {
    if (bx_hi[d] < bx_lo[d]) return reject(CAMR_ERR_INVALID, "empty box");
    if (uin->lo[d] > bx_lo[d] - NGROW || uin->hi[d] < bx_hi[d] + NGROW)
      return reject(CAMR_ERR_INVALID, "uin does not cover grow(bx, 4)");
    if (src && src->ptr && (src->lo[d] > bx_lo[d] - NGROW || src->hi[d] < bx_hi[d] + NGROW))
      return reject(CAMR_ERR_INVALID, "src does not cover grow(bx, 4)");
    if (dsdt->lo[d] > bx_lo[d] || dsdt->hi[d] < bx_hi[d])
      return reject(CAMR_ERR_INVALID, "dsdt does not cover bx");
  }
  if (uin->ncomp < NVAR || dsdt->ncomp < NVAR)
    return reject(CAMR_ERR_INVALID, "uin and dsdt need NVAR components");

  const bool mol = p->do_mol != 0;
  const bool has_src = src && src->ptr;
  Work w;
  w.s = make_space(bx_lo, bx_hi);
  const size_t need = work_doubles(w.s, mol, has_src, false) * sizeof(double);
  if (need > kScratchBytes) {
    std::snprintf(g_msg, sizeof(g_msg),
                  "box needs %zu bytes of scratch; the static scratch holds %zu bytes",
                  need, kScratchBytes);
    return CAMR_ERR_INVALID;
  }
  void* base = nullptr;
  const cudaError_t ea = scratch_address(static_cast<cudaStream_t>(stream), &base);
  if (ea != cudaSuccess) return cuda_status_of(ea);
  // Every scratch slot a call reads is written earlier in the same call
  // (each pass reads only the regions the previous passes produced), so no
  // clearing is needed between calls.
  work_carve(w, static_cast<double*>(base), mol, has_src, false);

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
  Lh.has_src = has_src;
  Lh.src = has_src ? make_dfab(*src) : Lh.uin;
  Lh.mol = mol;
  Lh.flx[0] = make_dfab(*flx0);
  Lh.flx[1] = make_dfab(*flx1);
  Lh.flx[2] = make_dfab(*flx2);
  Lh.dsdt = make_dfab(*dsdt);
  Lh.dt = DtRef{dt, nullptr};
  Lh.err = nullptr;
  return cuda_status_of(launch_hydro(Lh, w, static_cast<cudaStream_t>(stream)));
}
