/* camr_b200: B200-native (sm_100a) hydro advance for CAMR, C ABI.
 *
 * Every entry point takes plain pointers and sizes, returns a camr_status and
 * never aborts.  Device arrays use the Array4 layout of the reference:
 * component planes outermost, i fastest,
 *     idx = (i-lo0) + (j-lo1)*jstride + (k-lo2)*kstride + n*nstride.
 * State index layout (3-D, 3 species, Source/Utils/IndexDefines.H:17-83):
 *     URHO 0, UMX 1, UMY 2, UMZ 3, UEDEN 4, UEINT 5, UTEMP 6, UFS 7..9.
 * All arithmetic is FP64 and reproduces the reference bit for bit (the
 * library is built with -fmad=false; the reference CPU build uses
 * -ffp-contract=off).
 *
 * Streams are passed as `void*` holding a cudaStream_t (NULL = the legacy
 * default stream).  Work is stream-ordered; nothing synchronises the device
 * unless the entry point says so.
 */
#ifndef CAMR_B200_H
#define CAMR_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  CAMR_OK = 0,
  CAMR_ERR_INVALID = 1,       /* bad argument (null pointer, empty box, ...) */
  CAMR_ERR_UNSUPPORTED = 2,   /* parameter combination not implemented */
  CAMR_ERR_CUDA = 3,          /* a CUDA runtime call failed */
  CAMR_ERR_NUMERIC = 4,       /* device error word set (see camr_get_error) */
  CAMR_ERR_NOMEM = 5,         /* device allocation failed */
  CAMR_ERR_TIMEOUT = 6        /* a bounded device wait gave up */
} camr_status;

/* Boundary-condition words of CAMR.lo_bc / CAMR.hi_bc
 * (Source/Utils/IndexDefines.H:7-12). */
enum {
  CAMR_BC_INTERIOR = 0, CAMR_BC_INFLOW = 1, CAMR_BC_OUTFLOW = 2,
  CAMR_BC_SYMMETRY = 3, CAMR_BC_SLIPWALL = 4, CAMR_BC_NOSLIPWALL = 5
};

enum { CAMR_NVAR = 10, CAMR_QVAR = 11, CAMR_NQAUX = 5, CAMR_NGDNV = 6 };

/* The CAMR.* ParmParse parameters the hydro advance reads, by their
 * reference names (Source/Params/_cpp_parameters), plus eos_gamma (the
 * reference's compile-time EOS::gamma, Source/EOS/GammaLaw/EOS.H:16) and the
 * two constants of Source/Utils/CAMR_Constants.H:9-10.  camr_default_params
 * fills the reference defaults. */
typedef struct {
  int do_mol;
  int ppm_type;
  int plm_iorder;
  int use_pslope;
  int use_flattening;
  int transverse_reset_density;
  int dual_energy_update_E_from_e;
  int allow_negative_energy;
  int allow_small_energy;
  int add_grav_src;
  int riemann_solver;   /* 0 = the reference's two-shock solver (riemannus),
                           1 = HLLC (no counterpart in the reference; not
                           with embedded boundaries or the adjoint) */
  int eb_weights_type;  /* EB flux-redistribution weights (Hydro_utils_eb_K.H:
                           560-575): 0 one, 1 rho*(e + ke), 2 rho, 3 vfrac */
  double difmag;
  double small;
  double small_dens;
  double small_temp;
  double small_pres;
  double dual_energy_eta1;
  double dual_energy_eta2;
  double const_grav;
  double cfl;
  double init_shrink;
  double change_max;
  double fixed_dt;
  double initial_dt;
  double max_dt;
  double eos_gamma;
  double smallu;
  double small_num;
} camr_hydro_params;

/* Non-owning view of one Array4 on the device (AMReX FArrayBox::array()). */
typedef struct {
  double* ptr;
  int lo[3];
  int hi[3];
  int64_t jstride;
  int64_t kstride;
  int64_t nstride;
  int ncomp;
  int pad0;
} camr_fab;

/* Geometry of the level a box belongs to. */
typedef struct {
  int dom_lo[3];
  int dom_hi[3];
  int is_periodic[3];
  int bc_lo[3];
  int bc_hi[3];
  int pad0;
  double dx[3];
  double prob_lo[3];
} camr_geom;

/* Device error record (first failure wins). */
typedef struct {
  int code;      /* 0 none, 1 non-positive density/energy seen by ctoprim, 2 NaN,
                    3 density exactly zero in enforce_min_density, 4 index
                    out of range, 5 density below small_dens left unreset
                    (more cells below the floor in one pass than the reset
                    list holds: 16384) */
  int i, j, k;   /* cell of the first failure */
} camr_error_info;

/* Fill every default of Source/Params/_cpp_parameters. */
void camr_default_params(camr_hydro_params* p);

/* Library version string. */
const char* camr_version(void);

/* ---------------------------------------------------------------------
 * Per-box hydro: the drop-in for
 *   hydro_umdrv (Source/Hydro/Hydro.H:11-35, Source/Hydro/Hydro_umdrv.cpp:11-93)
 * together with the caller-side ctoprim/srctoprim launches of
 *   CAMR::construct_hydro_source (Source/Hydro/CAMR_construct_hydro_source.cpp:95-143).
 * uin: NVAR comps covering at least grow(bx,4), ghost cells filled and
 * cleaned (the reference's Sborder).  dsdt: NVAR on bx, ACCUMULATED (+=)
 * as the reference does.  flx[d]: NVAR on surroundingNodes(bx,d),
 * overwritten with the area-weighted fluxes (artificial viscosity included)
 * that feed the flux registers.  area[d]/vol may be NULL for Cartesian
 * metrics from geom->dx.  Temporaries come from a stream-ordered pool
 * (cudaMallocAsync), as the reference takes them from The_Async_Arena.
 * Sources: src may be NULL (zero sources); otherwise NVAR comps on the same
 * region as uin (the reference's sources_for_hydro).
 */
camr_status camr_hydro_umdrv(const int bx_lo[3], const int bx_hi[3],
                             const camr_geom* geom, const camr_fab* uin,
                             const camr_fab* src, camr_fab* dsdt,
                             camr_fab* flx0, camr_fab* flx1, camr_fab* flx2,
                             const camr_hydro_params* p, double dt,
                             void* stream);

/* The per-box hydro with the reference's full argument list
 * (Source/Hydro/Hydro.H:11-35): the caller supplies q (QVAR comps, the
 * reference's primitive layout Source/Utils/IndexDefines.H:54-59) and qaux
 * (NQAUX = 5 comps, :72-77) on grow(bx,4), as construct_hydro_source's
 * ctoprim computes them (Source/Hydro/CAMR_construct_hydro_source.cpp:
 * 108-120); src_q (QVAR comps on grow(bx,4), CTU only; NULL = zero) as
 * srctoprim computes them; and optionally the metric arrays: face areas
 * area[d] (1 comp on surroundingNodes(bx,d)) and cell volumes vol (1 comp
 * on bx) -- all four or none (none: Cartesian from geom->dx).  The
 * gamma-law EOS supplies QGAMC, QDPDR, QDPDE, QGAME and QTEMP, which are not
 * read.  uin (grow(bx,4)) is still read by the artificial viscosity.  dsdt
 * accumulated, flx overwritten, as camr_hydro_umdrv. */
camr_status camr_hydro_umdrv_full(const int bx_lo[3], const int bx_hi[3],
                                  const camr_geom* geom, const camr_fab* uin,
                                  const camr_fab* q, const camr_fab* qaux,
                                  const camr_fab* src_q, camr_fab* dsdt,
                                  camr_fab* flx0, camr_fab* flx1, camr_fab* flx2,
                                  const camr_fab* area0, const camr_fab* area1,
                                  const camr_fab* area2, const camr_fab* vol,
                                  const camr_hydro_params* p, double dt,
                                  void* stream);

/* ---------------------------------------------------------------------
 * Fab-level pieces of the level step for callers that keep their own box
 * loop (a CAMR build whose AMReX level driver stays and calls into this
 * library for parts of the step).  A level's data is a list of boxes, each
 * with a device fab (NVAR comps) covering the box grown by ng.  The boxes
 * must not overlap; they need not cover the domain (ghost cells whose
 * source no box holds are left alone, as at a coarse-fine boundary).
 * Stream-ordered; temporaries from cudaMallocAsync.
 */
typedef struct {
  int lo[3];
  int hi[3];
  camr_fab fab;
} camr_box_fab;

/* The single-level FillPatch of expand_state (Source/CAMR.cpp:1243-1250):
 * ng ghost layers of every fab from the valid cells of the boxes (interior
 * and periodic neighbours), past a physical boundary from the BC map of
 * Source/Utils/CAMR_setup.cpp:19-21 (foextrap and ext_dir copy the boundary
 * cell -- Exec/Sod's bcnormal -- reflect_even / reflect_odd mirror it). */
camr_status camr_fill_ghosts(const camr_geom* geom, int nbox, const camr_box_fab* boxes, int ng,
                             void* stream);
/* clean_state (Source/CAMR.cpp:1253-1262) of the boxes with ng ghost
 * layers: enforce_min_density on the valid cells (box by box in raster
 * order, each reset seen by the cells after it, as the reference's loop;
 * at most 16384 cells below the floor per call, else error code 5),
 * normalize_species on the valid cells, its FillBoundary of the interior
 * and periodic ghost cells, then computeTemp on every cell of the grown
 * boxes.  Errors go to the library's error word (camr_get_error). */
camr_status camr_clean_state(const camr_geom* geom, int nbox, const camr_box_fab* boxes, int ng,
                             const camr_hydro_params* p, void* stream);
/* The parts of camr_clean_state, for a caller whose boxes are spread over
 * processes and who exchanges ghost cells between them itself: clean_state
 * = CAMR_CLEAN_VALID (enforce_min_density + normalize_species on the valid
 * cells), then normalize_species' FillBoundary of the interior and periodic
 * ghost cells from the owners' normalized valid cells, then computeTemp on
 * every cell.  CAMR_CLEAN_GHOSTS_FROM_OWNERS does that FillBoundary for
 * ghosts whose owner is in the list and computeTemp on all ghost cells;
 * a distributed caller instead fills the interior ghosts itself after
 * CAMR_CLEAN_VALID and then asks for CAMR_CLEAN_GHOSTS_TEMP (computeTemp on
 * every ghost cell in place).  CAMR_CLEAN_VALID_TEMP: computeTemp on the
 * valid cells, which must come after every ghost fill has read them.
 * camr_clean_state = VALID | GHOSTS_FROM_OWNERS | VALID_TEMP. */
enum {
  CAMR_CLEAN_VALID = 1,
  CAMR_CLEAN_GHOSTS_FROM_OWNERS = 2,
  CAMR_CLEAN_GHOSTS_TEMP = 4,
  CAMR_CLEAN_VALID_TEMP = 8
};
camr_status camr_clean_state_parts(const camr_geom* geom, int nbox, const camr_box_fab* boxes,
                                   int ng, const camr_hydro_params* p, int parts, void* stream);
/* estTimeStep's hydro limit (Source/CAMR.cpp:490-563 with
 * Source/Utils/Timestep.H:18-61): cfl * the minimum over the valid cells of
 * dx_d / (c + |u_d|), capped by max_dt; fixed_dt when that is set.
 * Synchronises the stream. */
camr_status camr_est_dt(const camr_geom* geom, int nbox, const camr_box_fab* boxes,
                        const camr_hydro_params* p, double* dt, void* stream);
/* Read and clear the library's device error word on the current device
 * after the work queued on `stream` (synchronises it).  camr_hydro_umdrv and
 * camr_clean_state report into it where the reference would abort
 * (Source/Hydro/Hydro_ctoprim.H:56,68; Source/CAMR.cpp:997).  Returns
 * CAMR_ERR_NUMERIC when a failure was recorded. */
camr_status camr_get_error(void* stream, camr_error_info* info);

/* ---------------------------------------------------------------------
 * Batched per-box hydro over the boxes of one level (uneven sizes allowed):
 * the work-list form of the reference's MFIter box loop
 * (Source/Hydro/CAMR_construct_hydro_source.cpp:71-254).  Each task is one
 * box with its own fabs, exactly as for camr_hydro_umdrv; results are
 * identical to calling camr_hydro_umdrv box by box.
 */
typedef struct {
  int lo[3];
  int hi[3];
  camr_fab uin;     /* covers grow(box,4), ghost cells filled and cleaned */
  camr_fab src;     /* ptr NULL = zero sources */
  camr_fab dsdt;    /* on the box, accumulated */
  camr_fab flx[3];  /* on the box's faces, overwritten */
} camr_box_task;

typedef struct camr_batch camr_batch;

enum {
  CAMR_BATCH_PERSISTENT = 0,  /* one launch per stage for all boxes (work list) */
  CAMR_BATCH_PER_BOX = 1      /* the plain per-box launch sequence, box by box */
};

/* Build a plan: per-box workspaces (one device allocation) and the work-item
 * tables of every stage.  The fab pointers of the tasks are kept: run the
 * plan again after refilling the same fabs. */
camr_status camr_batch_create(int nbox, const camr_box_task* tasks,
                              const camr_geom* geom, const camr_hydro_params* p,
                              void* stream, camr_batch** out);
camr_status camr_batch_destroy(camr_batch* b);
/* Run the plan.  dt_dev (may be NULL) points to a device double read by the
 * kernels instead of dt, so a captured CUDA graph can follow a changing dt. */
camr_status camr_batch_run(camr_batch* b, double dt, const double* dt_dev,
                           int mode, void* stream);
/* Time each stage's candidates (cells per block 128/256/512; grid = one
 * block per work unit, or 1x / 2x the resident blocks of the device as a
 * persistent grid-stride launch) on the plan's own boxes and keep the
 * fastest.  Leaves dsdt untouched; synchronises. */
camr_status camr_batch_autotune(camr_batch* b, double dt, void* stream);
/* The chosen cells-per-block factor and grid of each stage (n >= 9). */
camr_status camr_batch_tuning(camr_batch* b, int* chunk, unsigned* grid, int n);
/* Set every stage's cells-per-block factor (1, 2 or 4: 128/256/512 cells) and
 * grid (0 = one block per work unit, else a persistent grid of that many
 * blocks), in camr_batch_tuning's order (n >= 9). */
camr_status camr_batch_set_tuning(camr_batch* b, const int* chunk, const unsigned* grid, int n);
/* One-shot convenience: create, run persistent, destroy (synchronises). */
camr_status camr_hydro_umdrv_batched(int nbox, const camr_box_task* tasks,
                                     const camr_geom* geom,
                                     const camr_hydro_params* p, double dt,
                                     void* stream);

/* ---------------------------------------------------------------------
 * Level-level API: one uniform level owned by the library on one GPU.
 * Replaces CAMR::CAMR_advance (Source/CAMR_advance.cpp:38-164) with its
 * construct_hydro_source box loop, expand_state/clean_state
 * (Source/CAMR.cpp:1243-1262), the gravity source Saxpys, post_timestep's
 * clean_state, and Amr's dt logic (estTimeStep/computeNewDt,
 * Source/CAMR.cpp:490-635).  The level's boxes are advanced as one padded
 * domain: results are identical for any box decomposition.
 */
typedef struct camr_level camr_level;

typedef struct {
  camr_geom geom;
  int max_grid_size[3];   /* box size of the level (enforce_min_density's
                             neighbour window); 0 = whole domain */
  int use_graph;          /* capture each step in a CUDA graph */
} camr_level_desc;

/* stream: the cudaStream_t the level issues its work on; NULL makes the
 * library create a non-blocking stream of its own (the legacy default
 * stream cannot be captured into a CUDA graph). */
camr_status camr_level_create(const camr_level_desc* desc,
                              const camr_hydro_params* p, void* stream,
                              camr_level** out);
camr_status camr_level_destroy(camr_level* lev);

/* Copy the valid-cell state in/out.  `state` holds NVAR comps on the
 * domain's valid cells, shape (NVAR, nz, ny, nx), i fastest.  host != 0:
 * the pointer is host memory (pinned for async); otherwise device memory. */
camr_status camr_level_set_state(camr_level* lev, const double* state, int host);
camr_status camr_level_get_state(camr_level* lev, double* state, int host);
/* Host transfers run on copy streams of their own: set_state(host) returns
 * once the upload is queued (the host buffer must stay unchanged until the
 * next camr_level_sync), and camr_level_get_state_async queues the download
 * without waiting for it.  Both overlap the level's kernels of neighbouring
 * steps.  camr_level_sync waits for all of the level's work and copies. */
camr_status camr_level_get_state_async(camr_level* lev, double* state, int host);
camr_status camr_level_sync(camr_level* lev);

/* CAMR::initData's epilogue: enforce_consistent_e then computeTemp. */
camr_status camr_level_init_finalize(camr_level* lev);

/* Restart (Amr::restart / CAMR::restart, Source/Utils/CAMR_io.cpp:23-43)
 * after camr_level_set_state with a checkpoint's state: dt_prev is the
 * checkpoint's dt_level and steps_done its level step count.  The next
 * step estimates the CFL dt from the restored state and applies
 * computeNewDt against dt_prev (change_max), as a run that never stopped
 * would, instead of computeInitialDt. */
camr_status camr_level_restart(camr_level* lev, double dt_prev, int steps_done);

/* Advance nsteps coarse steps.  The dt of each step is computed on the
 * device (first step: computeInitialDt; later: computeNewDt) unless
 * fixed_dts is non-NULL (host array of nsteps dts).  Stream-ordered; no
 * host synchronisation. */
camr_status camr_level_advance(camr_level* lev, int nsteps, const double* fixed_dts);

/* dt history / last dt (synchronises the level's stream). */
camr_status camr_level_last_dt(camr_level* lev, double* dt);
camr_status camr_level_est_dt(camr_level* lev, double* dt);

/* Take one (uncaptured) step with a CUDA event before every stage and
 * return each stage's device time in ms and its name (static strings).
 * Requires a previous step (the dt comes from computeNewDt). */
camr_status camr_level_profile_step(camr_level* lev, float* stage_ms,
                                    const char** names, int max_stages,
                                    int* nstages);

/* Kernel launches inside one graph-captured step (0 before the first
 * capture). */
int64_t camr_level_kernels_per_step(camr_level* lev);

/* The stream the level's work is issued on (for events / synchronisation). */
camr_status camr_level_stream(camr_level* lev, void** stream);

/* Device pointer to the padded state (domain grown by 4), and its layout. */
camr_status camr_level_state_fab(camr_level* lev, camr_fab* fab);

/* Read and clear the device error word (synchronises the level's stream). */
camr_status camr_level_get_error(camr_level* lev, camr_error_info* info);

/* Cells reset by enforce_min_density (Source/CAMR.cpp:941-1045) since the
 * level was created, counted over every clean_state of every step
 * (synchronises the level's stream).  Each cleaning pass of a step lists
 * the cells below small_dens and resets them in the reference's order: box
 * by box, in raster order, each reset visible to the cells after it.  At
 * most 16384 cells per pass; more set error code 5. */
camr_status camr_level_floor_resets(camr_level* lev, int64_t* cells);

/* ---------------------------------------------------------------------
 * Two-level AMR hierarchy (refinement ratio 2, subcycled): a base level
 * covering the domain and a fixed set of fine boxes.  Replaces, for two
 * levels, Amr::timeStep's recursion (level 0 advance, two level-1 substeps,
 * level 0 post_timestep) around CAMR::CAMR_advance
 * (Source/CAMR_advance.cpp:38-164): the fine level's FillPatch from its own
 * boxes and from the base level interpolated in time and space
 * (conservative linear), the flux register (CrseAdd / FineAdd,
 * Source/Hydro/CAMR_construct_hydro_source.cpp:243-254) and its reflux,
 * avgDown and the coarse clean_state of post_timestep
 * (Source/CAMR.cpp:679-718, :803-851, :1048-1066), and computeNewDt /
 * computeInitialDt over both levels (:566-676).  Periodic domains; the box
 * layout stays fixed (no regridding).
 */
typedef struct camr_amr camr_amr;

/* base: the level-0 description (domain, max_grid_size, use_graph).
 * boxes: nbox fine boxes, each lo0,lo1,lo2,hi0,hi1,hi2 in the fine index
 * space; every lo even and every hi odd (whole coarse cells), inside the
 * fine domain, not overlapping.  stream as for camr_level_create. */
camr_status camr_amr_create(const camr_level_desc* base, int nbox, const int* boxes,
                            const camr_hydro_params* p, void* stream, camr_amr** out);
camr_status camr_amr_destroy(camr_amr* a);

/* Copy the states in/out: S0 the base level's valid cells (NVAR, nz, ny,
 * nx); S1 the fine boxes' valid cells, box after box, each (NVAR, nz, ny,
 * nx).  host != 0: host pointers.  set_state resets the clock: the next
 * step starts at time 0 with computeInitialDt. */
camr_status camr_amr_set_state(camr_amr* a, const double* S0, const double* S1, int host);
camr_status camr_amr_get_state(camr_amr* a, double* S0, double* S1, int host);

/* CAMR::initData's epilogue on both levels, then post_init's avgDown. */
camr_status camr_amr_init_finalize(camr_amr* a);

/* Advance nsteps coarse steps (each: one base step, two fine substeps,
 * reflux, average down).  Stream-ordered; after the first step every step
 * replays one CUDA graph when use_graph is set. */
camr_status camr_amr_advance(camr_amr* a, int nsteps);

/* clock[0..3]: time of level 0, time of level 1, last dt of level 0, last
 * dt of level 1 (synchronises). */
camr_status camr_amr_clock(camr_amr* a, double clock[4]);

/* Restart after camr_amr_set_state with a checkpoint's states: clock as
 * camr_amr_clock returns it (times and last dts of both levels) and the
 * coarse steps done.  The next coarse step estimates the CFL dt of both
 * levels from the restored states and applies computeNewDt against the
 * checkpoint's dts, as an uninterrupted run would (synchronises). */
camr_status camr_amr_restart(camr_amr* a, const double clock[4], int steps_done);

/* Cells enforce_min_density has reset on either level since the hierarchy
 * was created (synchronises).  Every cleaning pass of both levels lists the
 * cells below small_dens and resets them in the reference's order, each
 * box of a level its own window (the fine boxes, the base level's
 * max_grid_size boxes); post_timestep's clean of level 0 follows reflux and
 * avgDown.  At most 16384 cells per pass; more set error code 5. */
camr_status camr_amr_floor_resets(camr_amr* a, int64_t* cells);

/* Autotune the fine level's batched hydro on its current state (after at
 * least one step); synchronises. */
camr_status camr_amr_autotune(camr_amr* a);

/* How the fine level's hydro is issued: CAMR_BATCH_PERSISTENT (default:
 * one work-list launch per stage for all boxes, the step graph-captured) or
 * CAMR_BATCH_PER_BOX (the plain per-box launch sequences, box by box, as
 * the reference's MFIter loop issues them; no graph).  Same results. */
camr_status camr_amr_set_fine_mode(camr_amr* a, int mode);

/* Number of fine cells (valid) and kernel launches inside one captured
 * coarse step (0 before the first capture). */
int64_t camr_amr_fine_cells(camr_amr* a);
int64_t camr_amr_kernels_per_step(camr_amr* a);
camr_status camr_amr_stream(camr_amr* a, void** stream);

/* Read and clear the device error word of both levels (synchronises). */
camr_status camr_amr_get_error(camr_amr* a, camr_error_info* info);

/* ---------------------------------------------------------------------
 * Discrete adjoint of the MOL level step (SSP-RK2, PLM slopes, two-shock
 * Riemann; periodic uniform level, do_mol = 1, default energy flags).  No
 * counterpart in the reference: it differentiates the CAMR_advance MOL
 * path (Source/CAMR_advance.cpp:124-136 and what it calls) by hand, step by
 * step in reverse, with the dt sequence of the forward pass frozen and
 * checkpoint-and-recompute over time steps.
 */
typedef struct camr_adjoint camr_adjoint;

camr_status camr_adjoint_create(const camr_geom* geom, const camr_hydro_params* p,
                                int checkpoint_every, void* stream, camr_adjoint** out);
camr_status camr_adjoint_destroy(camr_adjoint* a);
/* Forward nsteps steps from S0 to S_final (device pointers, valid cells
 * (NVAR, nz, ny, nx)).  dt per step: computeInitialDt / computeNewDt on the
 * device, or the host array fixed_dts.  Keeps a checkpoint every
 * checkpoint_every steps and the dt sequence for the backward pass. */
camr_status camr_adjoint_forward(camr_adjoint* a, const double* S0, double* S_final,
                                 int nsteps, const double* fixed_dts);
/* Adjoint of the last forward run: lam0 = (dS_final/dS0)^T lam_final
 * (device pointers, same layout).  UTEMP carries no adjoint (no other
 * state variable depends on it). */
camr_status camr_adjoint_backward(camr_adjoint* a, const double* lam_final, double* lam0);
/* The dt sequence of the last forward run (synchronises). */
camr_status camr_adjoint_dts(camr_adjoint* a, double* dts, int n);
camr_status camr_adjoint_stream(camr_adjoint* a, void** stream);
camr_status camr_adjoint_get_error(camr_adjoint* a, camr_error_info* info);

/* ---------------------------------------------------------------------
 * Embedded-boundary per-box hydro: hydro_umdrv_eb
 * (Source/Hydro/Hydro_umdrv_eb.cpp:14-191), MOL (MOL_umeth_eb) or, with
 * do_mol = 0, Godunov-PLM (Godunov_umeth_eb, ppm_type must be 0; zero
 * predictor sources), with flux redistribution (AMReX's FluxRedist,
 * restated).  ng = 5 for MOL, 6 for Godunov.  Geometry on a cell region G
 * covering grow(bx, ng), device pointers, i fastest:
 *   flag   G cells: bits 0-1 type (0 regular, 1 cut, 3 covered), bit
 *          2 + (di+1) + 3 (dj+1) + 9 (dk+1) connectivity to neighbour
 *          (di,dj,dk) (the cell itself included)
 *   vfrac  G cells; ap[d] faces of G in direction d (surroundingNodes(G, d));
 *   fc[d]  2 components (transverse directions in x, y, z order) on the
 *          same faces, component planes outermost.
 * uin covers grow(bx, ng).  dsdt (bx) is overwritten (the reference's
 * redistribution writes it); flx[d] receive the face-centroid fluxes of
 * bx's faces.  redist: 1 = flux redistribution, 0 = none, 2 = state
 * redistribution (Berger & Giuliani's method, restated: AMReX's own is not
 * the reference's code; ng grows by one).
 */
typedef struct {
  const unsigned* flag;
  const double* vfrac;
  const double* ap[3];
  const double* fc[3];
  int g_lo[3];
  int g_hi[3];
  const double* cent;  /* cell-centroid offsets, 3 comps on G (may be NULL:
                          cell centres); read by state redistribution */
} camr_eb_geom;

camr_status camr_hydro_umdrv_eb(const int bx_lo[3], const int bx_hi[3], const camr_geom* geom,
                                const camr_fab* uin, const camr_eb_geom* eb, camr_fab* dsdt,
                                camr_fab* flx0, camr_fab* flx1, camr_fab* flx2,
                                const camr_hydro_params* p, int redist, double dt,
                                void* stream);

/* ---------------------------------------------------------------------
 * EB level: one uniform level with an embedded boundary, MOL or Godunov-PLM
 * (CAMR_advance, Source/CAMR_advance.cpp:38-164, with hydro_umdrv_eb per
 * stage and the EB build's clean_state / computeTemp / estTimeStep guards
 * for covered cells), 5 ghost cells for MOL, 6 for Godunov.  desc->max_grid_size
 * chops the domain into boxes (0 = one box): as in an EB build's
 * construct_hydro_source, covered boxes are skipped, boxes whose grow(box,2)
 * (grow(box,3) with state redistribution) is all regular run the regular
 * hydro (one batched launch per stage for all of them) and the others the
 * EB hydro.  eb: geometry over exactly grow(domain, ng), host or device
 * memory, copied into the level; ng = 5 for MOL, 6 for Godunov, one more
 * with state redistribution.  Godunov requires ppm_type = 0
 * (Source/CAMR.cpp:186-190) and no gravity source.  redist: 0 NoRedist,
 * 1 FluxRedist, 2 StateRedist (restated method).  Covered cells hold zero
 * state (initData's EB_set_covered); set_state/get_state/advance/dts as
 * for camr_level_*.
 */
typedef struct camr_eb_level camr_eb_level;

camr_status camr_eb_level_create(const camr_level_desc* desc, const camr_eb_geom* eb,
                                 const camr_hydro_params* p, int redist, void* stream,
                                 camr_eb_level** out);
camr_status camr_eb_level_destroy(camr_eb_level* lev);
camr_status camr_eb_level_set_state(camr_eb_level* lev, const double* state, int host);
camr_status camr_eb_level_get_state(camr_eb_level* lev, double* state, int host);
/* initData's epilogue with the EB guards: enforce_consistent_e where rho > 0,
 * computeTemp (T = 0 where rho <= 0). */
camr_status camr_eb_level_init_finalize(camr_eb_level* lev);
camr_status camr_eb_level_advance(camr_eb_level* lev, int nsteps, const double* fixed_dts);
/* The dt of every step taken since creation (at most n), and their count. */
camr_status camr_eb_level_dts(camr_eb_level* lev, double* dts, int n, int* nsteps);
/* Tune the launch shapes of the regular boxes' batched stages on the
 * level's current Sborder; call after a step.  Each stage is first timed
 * alone (camr_batch_autotune); then whole hydro stages, regular and cut boxes
 * running together as one captured graph, are timed with that choice, with
 * the same choice on non-persistent grids, and with the untuned shapes, and
 * the fastest is kept.  Synchronises. */
camr_status camr_eb_level_autotune(camr_eb_level* lev);
/* How the level's boxes were classified: all-regular grow(box,2) (regular
 * hydro), cut (EB hydro), covered (skipped). */
camr_status camr_eb_level_boxes(camr_eb_level* lev, int* regular, int* cut, int* covered);
int64_t camr_eb_level_kernels_per_step(camr_eb_level* lev);
camr_status camr_eb_level_stream(camr_eb_level* lev, void** stream);
camr_status camr_eb_level_get_error(camr_eb_level* lev, camr_error_info* info);
/* Cells enforce_min_density has reset since the level was created
 * (synchronises).  As camr_level_floor_resets, with the EB build's guard:
 * covered cells are never reset, but they are neighbours like any other
 * cell (Source/CAMR.cpp:960-1043). */
camr_status camr_eb_level_floor_resets(camr_eb_level* lev, int64_t* cells);

/* ---------------------------------------------------------------------
 * Plotfile output / input of one level (host memory), in AMReX's plotfile
 * layout as CAMR::writePlotFile writes it (Source/Utils/CAMR_io.cpp:408-565):
 * dir/Header, dir/Level_0/Cell_H (VisMF header), dir/Level_0/Cell_D_00000
 * (one FAB per box, little-endian IEEE doubles).  state: NVAR comps on the
 * domain's valid cells, shape (NVAR, nz, ny, nx), i fastest.  boxes: nbox
 * boxes as lo0,lo1,lo2,hi0,hi1,hi2 (the level's grids).  comps (may be
 * NULL = 0..ncomp-1) selects the state components written and names (may
 * be NULL) their plot names (default: the reference's state names,
 * Source/Utils/CAMR_setup.cpp:159-198).  geom supplies the domain, dx and
 * prob_lo.  camr_read_plotfile reads the ncomp written components back into
 * the first ncomp planes of state (single-level plotfiles).
 */
camr_status camr_write_plotfile(const char* dir, const camr_geom* geom, const double prob_hi[3],
                                double time, int level_step, int nbox, const int* boxes,
                                const double* state, int ncomp, const int* comps,
                                const char* const* names);
camr_status camr_read_plotfile(const char* dir, const camr_geom* geom, int ncomp,
                               double* state, double* time, int* level_step);
/* The two levels of the AMR driver (camr_amr_*, refinement ratio 2) as one
 * plotfile, as CAMR::writePlotFile writes a two-level hierarchy: level 0 as
 * above (geom, boxes0, state0); level 1 on the fine index space (domain
 * 2*dom_lo .. 2*dom_hi+1, cell size dx/2), nbox1 boxes (lo0,lo1,lo2,
 * hi0,hi1,hi2) whose states lie back to back in state1, each
 * (NVAR, nz, ny, nx) over its own box (the layout of camr_amr_get_state).
 * level_step[2]: the step counts of the two levels.  nbox1 = 0 writes a
 * single-level plotfile. */
camr_status camr_write_plotfile_amr(const char* dir, const camr_geom* geom, const double prob_hi[3],
                                    double time, const int level_step[2], int nbox0,
                                    const int* boxes0, const double* state0, int nbox1,
                                    const int* boxes1, const double* state1, int ncomp,
                                    const int* comps, const char* const* names);
/* Reads a plotfile of camr_write_plotfile_amr back: level 0 into state0
 * (first ncomp planes), level 1 into state1 laid out as for the writer; the
 * file's fine boxes must be boxes1 in the same order (a restart of the same
 * hierarchy).  level_step (may be NULL) receives both levels' steps. */
camr_status camr_read_plotfile_amr(const char* dir, const camr_geom* geom, int ncomp,
                                   double* state0, int nbox1, const int* boxes1,
                                   double* state1, double* time, int level_step[2]);
/* Checkpoint of one level or of the two-level hierarchy, in the layout of
 * CAMR::checkPoint (Source/Utils/CAMR_io.cpp:45-60), i.e. AMReX's
 * Amr::checkPoint with AmrLevel / StateData records: dir/Header (times,
 * dt_level, n_cycle, level steps, per-level geometry, BoxArray and state
 * record), Level_L/SD_0_New_MF_H and _D_00000 (VisMF, NVAR comps, the new
 * state), and dir/CPUtime.  time[l], dt[l], level_step[l]: each level's
 * time, last dt and step count.  Level 0: nbox0 boxes (lo0,lo1,lo2,hi0,
 * hi1,hi2) with state0 over the domain (NVAR, nz, ny, nx); level 1 (nbox1 =
 * 0: none) as for camr_write_plotfile_amr.  AMReX is not present here, so
 * its own restart reader has not read these files. */
camr_status camr_write_checkpoint(const char* dir, const camr_geom* geom, const double prob_hi[3],
                                  const double time[2], const double dt[2],
                                  const int level_step[2], int nbox0, const int* boxes0,
                                  const double* state0, int nbox1, const int* boxes1,
                                  const double* state1, double cpu_time);
/* Reads a checkpoint of camr_write_checkpoint back: times, dts, steps and
 * the states (level 1 for the same fine boxes in the same order). */
camr_status camr_read_checkpoint(const char* dir, const camr_geom* geom, double time[2],
                                 double dt[2], int level_step[2], double* state0, int nbox1,
                                 const int* boxes1, double* state1);

/* Why the last plotfile call on this thread failed ("" if it did not). */
const char* camr_io_last_error(void);

/* ---------------------------------------------------------------------
 * Allocation-free per-box hydro.  No counterpart in the reference: it is
 * camr_hydro_umdrv for callers that may not allocate device memory while
 * they run (code inside an arena or pool that owns all device memory,
 * real-time loops that forbid allocator calls after start-up, hosts where
 * cudaMalloc/cudaMallocAsync would fight another allocator).  Same
 * arguments and results as camr_hydro_umdrv; the scratch is a fixed
 * CAMR_NOALLOC_SCRATCH_BYTES array in device memory, which every GPU that
 * loads the library keeps until the process exits.  It holds a CTU box of
 * up to 28^3 cells or a MOL box of up to 49^3 without a source fab (CTU up
 * to 27^3 with one).  Boxes whose scratch does not fit are rejected with
 * CAMR_ERR_INVALID, and parameters exactly as camr_hydro_umdrv rejects them
 * (camr_noalloc_last_error says why).  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress); make that first call before any stream
 * capture.  All calls share the one array: calls that overlap on the GPU
 * race on it and must be serialised by the caller.  Calls no cudaMalloc,
 * cudaFree or allocating library routine.
 */
#define CAMR_NOALLOC_SCRATCH_BYTES (64u * 1024u * 1024u)
camr_status camr_hydro_umdrv_noalloc(const int bx_lo[3], const int bx_hi[3],
                                     const camr_geom* geom, const camr_fab* uin,
                                     const camr_fab* src, camr_fab* dsdt,
                                     camr_fab* flx0, camr_fab* flx1,
                                     camr_fab* flx2, const camr_hydro_params* p,
                                     double dt, void* stream);

/* Why the last camr_hydro_umdrv_noalloc call on this thread was rejected
 * ("" if it was not). */
const char* camr_noalloc_last_error(void);

/* Text of the last CUDA error this thread saw in the library ("" if none). */
const char* camr_last_error_string(void);

/* Measure the FP64 FMA throughput of the device with independent DFMA
 * chains (a roofline denominator); synchronises.  Result in TFLOP/s. */
camr_status camr_measure_fp64_peak(double* tflops, void* stream);

/* Check the kernels' shared-reciprocal quotient (a / b from RN(1/b) with
 * fused multiply-add corrections) against the device's IEEE division on
 * about 5 n operand pairs (random, next to rounding midpoints, integer
 * ratios, special values); *mismatches counts the pairs whose bits differ
 * (synchronises). */
camr_status camr_check_rn_div(int64_t n, uint64_t seed, int64_t* mismatches, void* stream);

/* Kernel launches issued by the library so far (for accounting; graph
 * replays count the kernels they contain). */
int64_t camr_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif
