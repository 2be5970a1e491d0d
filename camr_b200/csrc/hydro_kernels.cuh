// Kernels of the per-box hydro right-hand side and their launcher.
//
// Work decomposition (CTU, the reference's Godunov_umeth):
//   K1 ctoprim        cells of grow(bx,4)            -> Q (+ SRCQ)
//   K2 flatten/divu   cells of grow(bx,1)            -> FLAT, DIVU on nodes of bx
//   K3 trace          (cell of grow(bx,1), dir)      -> SM[d], SP[d] face states
//   K4 flux1          (E-face, E)                    -> F1[E], BC edits of SM/SP
//   K5 flux2          (D-face, D|E combination)      -> F2[D|E]
//   K6 flux3          (F-face of bx, F)              -> flx[F] (caller), QF[F]
//   K7 consup         cells of bx                    -> dsdt += ...
// MOL (MOL_umeth): K1, K2 (divu only), slopes per (cell, dir), one face
// pass (edge states + Riemann + adjust), K7.
// Every face flux is computed once, on exactly the faces whose value reaches
// the box's fluxes and dsdt.
#pragma once

#include "hydro_point.cuh"

namespace camr {

// dt either as a value or read from device memory (the level driver keeps
// the dt sequence on the device so a whole step can be graph-captured).
struct DtRef {
  double v;
  const double* p;
  __device__ __forceinline__ double get() const { return p ? *p : v; }
};

// Intermediate arrays of one box, all indexed in the box's Space.
struct Work {
  Space s;
  double* q;        // SQ_N comps
  double* srcq;     // ES_N comps (only with sources)
  double* flat;     // 1 comp
  double* divu;     // 1 comp (nodes)
  double* sm[3];    // ES_N comps each (minus state on d-faces)
  double* sp[3];    // ES_N comps each (plus state on d-faces)
  double* f1[3];    // FR_N comps each
  double* f2[6];    // FR_N comps each, index combo(D,E)
  double* qf[3];    // 2 comps each: interface pressure, normal velocity
  double* slope[3]; // MOL slope layout: 8 comps each (split layout: sm/sp hold
                    // the ML_* left pieces / right edge states instead)
};

// Combination index of the second-pass "D|E" fluxes.
__host__ __device__ constexpr int combo(int D, int E) {
  return D * 2 + ((E > D) ? E - 1 : E);
}

// mol_split = false: the MOL slope layout (slope[d]) instead of the edge
// states of the split cell/face passes (sm[d], sp[d]) -- smaller, and what
// a slope tape needs.
size_t work_doubles(const Space& s, bool mol, bool has_src, bool mol_split = true);
void work_carve(Work& w, double* base, bool mol, bool has_src, bool mol_split = true);

// Optional per-stage event marks (profiling): mark() records the next event
// on the launch stream before a stage is issued.
struct StageTimer {
  static constexpr int kMax = 40;
  cudaEvent_t ev[kMax];
  const char* name[kMax];
  int n = 0;
  void mark(cudaStream_t st, const char* what) {
    if (n < kMax) {
      name[n] = what;
      cudaEventRecord(ev[n++], st);
    }
  }
};

// Caller-supplied metric arrays of the reference's hydro_umdrv (Source/
// Hydro/Hydro.H:11-35): face areas a[d] on surroundingNodes(bx,d) and cell
// volumes on bx.  on = 0: Cartesian metrics from dx (the default).
struct Metrics {
  DFab a[3];
  DFab vol;
  int on = 0;
};

struct HydroLaunch {
  KGeom g;
  KParams P;
  DFab uin;
  DFab src;        // valid when has_src
  bool has_src;
  bool mol;
  DFab flx[3];     // caller flux fabs (faces of bx)
  DFab dsdt;       // caller dsdt (bx), accumulated
  DtRef dt;
  DevError* err;
  StageTimer* timer = nullptr;
  // Caller-supplied primitive state (QVAR comps), qaux (NQAUX) and
  // primitive sources (QVAR) on grow(bx,4), in the reference's layout,
  // used instead of ctoprim / srctoprim (ext_q; srcq only with ext_srcq).
  bool ext_q = false;
  bool ext_srcq = false;
  DFab qin, qauxin, srcqin;
  Metrics M;
  // MOL: keep the slopes in Work::slope (the adjoint's tape reads them);
  // otherwise slopes and faces run fused and the slope arrays stay unused
  bool keep_slopes = false;
};

// ---- batched (work-list) launches over many boxes of one level ----
enum { BS_CTOPRIM = 0, BS_FLATDIVU, BS_TRACE, BS_FLUX1, BS_FLUX2, BS_FLUX3, BS_MOLSLOPE,
       BS_MOLFLUX, BS_CONSUP, BS_COUNT };

// Everything one box of a batch needs on the device.
struct BoxCtx {
  KGeom g;
  Work w;
  DFab uin, src;
  DFab flx[3];
  DFab dsdt;
  bool has_src;
  bool mol;
  // EB cell flags over [eblo, eblo + ebn) (null outside an EB level):
  // ctoprim leaves q = 0 in covered cells, as construct_hydro_source does
  // in an EB build (CAMR_construct_hydro_source.cpp:108-120).
  const unsigned* ebflag;
  int eblo[3], ebn[3];
};

// One work item of a batched stage: `region` of box `box` in sub-direction
// `sub`, starting at global block `block0`.
struct BatchItem {
  int64_t block0;
  Region r;
  int box;
  int sub;
};

int stage_regions(int stage, const KGeom& g, Region* out);
// bitem: the item of each of the nblocks blocks (or null: each block
// binary-searches the items' first blocks).
cudaError_t launch_batched_stage(int stage, const BoxCtx* boxes, const BatchItem* items,
                                 int nitems, const int* bitem, int64_t nblocks, int chunk,
                                 unsigned grid, const KParams& P, DtRef dt, DevError* err,
                                 cudaStream_t st);
const void* batched_kernel(int stage);
int batched_min_blocks(int stage);
constexpr int kBatchBlock = 128;

// A batch plan whose stages stop at the face fluxes (flx and the interface
// p, u_n of each box's Work): the caller forms the update itself.  The
// tasks' dsdt fabs are not used.  Run with camr_batch_run.
camr_status batch_create_fluxes(int nbox, const camr_box_task* tasks, const camr_geom* geom,
                                const camr_hydro_params* p, cudaStream_t st, camr_batch** out);
const Work& batch_work(const camr_batch* b, int box);

// A full batch plan (dsdt accumulated) for the regular boxes of an EB level:
// ctoprim skips the covered cells of the flag array over [glo, glo + gn).
camr_status batch_create_eb(int nbox, const camr_box_task* tasks, const camr_geom* geom,
                            const camr_hydro_params* p, cudaStream_t st, const unsigned* flag,
                            const int glo[3], const int gn[3], camr_batch** out);

// Issue the whole per-box hydro on `stream` (7 or 5 kernel launches).
cudaError_t launch_hydro(const HydroLaunch& L, const Work& w, cudaStream_t stream);

// Pieces reused by the level driver.
cudaError_t launch_hydro_fluxes(const HydroLaunch& L, const Work& w, cudaStream_t stream);

}  // namespace camr
