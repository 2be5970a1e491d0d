/* C interface of the CPU oracle libraries (test infrastructure only).
 *
 * Two shared libraries export exactly this interface:
 *   oracle/_lib/libcamr_oracle.so  - the repo's CPU restatement of CAMR's
 *                                    hydro advance (oracle/hydro_restate.cpp)
 *   oracle/_ref/libcamr_ref.so     - the reference's own per-box hydro sources
 *                                    (Source/Hydro/**) compiled against the
 *                                    AMReX stand-in in oracle/amrex_shim
 * Both link the same restated level driver (oracle/level_driver.cpp), so a
 * whole run differs between them only in the per-box hydro arithmetic.
 *
 * Layout of every array: Array4 order, component planes outermost, i fastest:
 *   idx = (i-lo0) + (j-lo1)*nx + (k-lo2)*nx*ny + n*nx*ny*nz
 * State index layout (3-D, 3 species): URHO 0, UMX 1, UMY 2, UMZ 3, UEDEN 4,
 * UEINT 5, UTEMP 6, UFS 7..9 (Source/Utils/IndexDefines.H:17-83).
 */
#ifndef CAMR_ORACLE_ABI_H
#define CAMR_ORACLE_ABI_H

#ifdef __cplusplus
extern "C" {
#endif

/* Boundary-condition words of CAMR.lo_bc / CAMR.hi_bc
 * (Source/Utils/IndexDefines.H:7-12). */
enum { ORC_INTERIOR = 0, ORC_INFLOW = 1, ORC_OUTFLOW = 2, ORC_SYMMETRY = 3,
       ORC_SLIPWALL = 4, ORC_NOSLIPWALL = 5 };

/* Every CAMR.* ParmParse parameter the hydro advance reads
 * (Source/Params/_cpp_parameters), plus eos_gamma (EOS.H:16 holds it as a
 * compile-time 1.4) and the two CAMRConstants (Utils/CAMR_Constants.H:9-10). */
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
  int eb_weights_type;  /* EB flux-redistribution weights (default 2 = rho) */
  int riemann_solver;   /* 0 riemannus (the reference); 1 HLLC (restatement
                           only: the reference has no such option) */
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
  double smallu;    /* CAMRConstants::smallu = 1e-12 */
  double small_num; /* CAMRConstants::small_num = 1e-8 */
} orc_params;

/* One level of a uniform grid: the domain, its boundary words and the box
 * decomposition (boxes of max_grid_size, cut into hydro tiles of tile_size;
 * a zero tile size means one tile per box). */
typedef struct {
  int dom_lo[3];
  int dom_hi[3];
  int is_periodic[3];
  int bc_lo[3];
  int bc_hi[3];
  int max_grid_size[3];
  int tile_size[3];
  int nthreads;
  double dx[3];
} orc_level;

/* Per-box hydro: one MFIter iteration of CAMR::construct_hydro_source.
 * uin covers at least grow(bx,4) (uin_lo/uin_hi); src likewise or NULL
 * (= zero sources); dsdt covers bx and is accumulated; flx[d] cover
 * surroundingNodes(bx,d) and are overwritten; area/vol may be NULL (uniform
 * Cartesian metrics from dx).  Returns the count of assertion failures the
 * reference kernels reported (0 on success). */
long orc_hydro_box(const orc_params* p, const int bx_lo[3], const int bx_hi[3],
                   const int dom_lo[3], const int dom_hi[3], const int bclo[3],
                   const int bchi[3], const double* uin, const int uin_lo[3],
                   const int uin_hi[3], const double* src, double* dsdt,
                   const int dsdt_lo[3], const int dsdt_hi[3], double* flx0,
                   double* flx1, double* flx2, const double dx[3], double dt);

/* oracle/_ref only: the reference's hydro_ctoprim + hydro_srctoprim over
 * [lo, hi] of uin (src NULL = zero sources): q (QVAR), qaux (NQAUX) and
 * src_q (QVAR) on that region. */
long orc_ref_ctoprim(const orc_params* p, const int lo[3], const int hi[3], const double* uin,
                     const int uin_lo[3], const int uin_hi[3], const double* src, double* q,
                     double* qaux, double* srcq);

/* oracle/_ref only: the reference's hydro_umdrv with caller q, qaux (and
 * src_q, NULL = zero) on grow(bx,4) and caller face areas / volumes (NULL
 * = Cartesian from dx); flx overwritten, dsdt (on bx) accumulated. */
long orc_ref_hydro_box_full(const orc_params* p, const int bx_lo[3], const int bx_hi[3],
                            const int dom_lo[3], const int dom_hi[3], const int bclo[3],
                            const int bchi[3], const double* uin, const int uin_lo[3],
                            const int uin_hi[3], const double* q, const double* qaux,
                            const double* srcq, const double* area0, const double* area1,
                            const double* area2, const double* vol, double* dsdt,
                            double* flx0, double* flx1, double* flx2, const double dx[3],
                            double dt);

/* oracle/_ref/libcamr_ref_flops.so only: the reference's per-box hydro on
 * the box [0, n-1] (uin: NVAR comps on grow(bx,4), zero sources, Cartesian
 * metrics) with counted operations: counts = adds, multiplies, divides,
 * square roots, comparisons, abs/copysign. */
long orc_count_flops(const orc_params* p, const int n[3], const int bclo[3], const int bchi[3],
                     const double* uin, const double dx[3], double dt, long long counts[6]);

/* Fill every ParmParse default of the reference (Source/Params/_cpp_parameters). */
void orc_default_params(orc_params* p);

/* Problem initialisation epilogue of CAMR::initData (Source/CAMR.cpp:414-420):
 * enforce_consistent_e then computeTemp on the valid cells. */
void orc_init_finalize(const orc_params* p, const orc_level* lev, double* state);

/* CAMR::estTimeStep (Source/CAMR.cpp:490-563) on the valid state. */
double orc_est_dt(const orc_params* p, const orc_level* lev, const double* state);

/* Advance `nsteps` coarse steps of a single-level run, each one
 * Amr::coarseTimeStep -> computeNewDt/computeInitialDt -> CAMR::advance ->
 * post_timestep.  state: NVAR comps on the valid domain, updated in place.
 * dt_prev: in = dt of the previous step (ignored when first_step), out = the
 * last dt taken.  dt_hist (may be NULL) receives every dt.  Returns 0 or the
 * number of assertion failures seen. */
long orc_advance(const orc_params* p, const orc_level* lev, double* state,
                 int nsteps, int first_step, double* dt_prev, double* dt_hist);

/* Same as orc_advance but with a fixed, caller-given dt sequence. */
long orc_advance_fixed_dt(const orc_params* p, const orc_level* lev,
                          double* state, int nsteps, const double* dts);

/* FillPatch + clean_state of one padded copy (the domain grown by ng): the
 * border state the hydro of a level step reads (Source/CAMR.cpp:1243-1262). */
void orc_expand_state(const orc_params* p, const orc_level* lev,
                      const double* state, int ng, double* border);

/* Two-level AMR run (refinement ratio 2, subcycling, reflux, average
 * down; periodic domains).  lev0: the base level.  boxes: nbox fine boxes
 * as lo0,lo1,lo2,hi0,hi1,hi2 in the fine index space (coarse-aligned).
 * S0: base state (valid cells); S1: the fine boxes' states, box after box,
 * each (NVAR, nz, ny, nx).  do_init: apply initData's epilogue to both
 * levels and post_init's average-down first.  first_step: take the
 * first dt from computeInitialDt.  clock (in/out): time of level 0, time
 * of level 1, last dt of level 0, last dt of level 1.  dt_hist (may be
 * NULL): 2*nsteps doubles, the dt of each level per coarse step. */
long orc_amr_run(const orc_params* p, const orc_level* lev0, int nbox, const int* boxes,
                 double* S0, double* S1, int nsteps, int do_init, int first_step,
                 double* clock, double* dt_hist);

/* Per-box EB hydro, MOL (oracle/_ref/libcamr_ref_eb.so only): the
 * reference's EB kernels (hydro_ctoprim, MOL_umeth_eb, adjust_fluxes_eb,
 * hydro_consup_eb) in hydro_umdrv_eb's order, then flux redistribution
 * (redist = 1, restated) or none (redist = 0).  uin, flag, vfrac cover G =
 * [g_lo, g_hi] (at least grow(bx, 5)); ap[d] and fc[d] (2 comps) cover
 * surroundingNodes(G, d).  flag: bits 0-1 type (0 regular, 1 cut, 3
 * covered), bit 2 + (di+1) + 3(dj+1) + 9(dk+1) connectivity; cent (3 comps,
 * may be NULL = cell centres) the cell-centroid offsets.  redist: 0 none,
 * 1 flux redistribution, 2 state redistribution (one more ghost layer:
 * G at least grow(bx, 6) for MOL, 7 for Godunov).  dsdt (bx) is
 * overwritten; flx[d] receive the face-centroid fluxes of bx's faces. */
long orc_hydro_box_eb(const orc_params* p, const int bx_lo[3], const int bx_hi[3],
                      const int dom_lo[3], const int dom_hi[3], const int bclo[3],
                      const int bchi[3], const int periodic[3], const double* uin,
                      const int g_lo[3], const int g_hi[3], const unsigned* flag,
                      const double* vfrac, const double* ap0, const double* ap1,
                      const double* ap2, const double* fc0, const double* fc1, const double* fc2,
                      const double* cent, int redist, int weights_type, double* dsdt,
                      double* flx0, double* flx1, double* flx2, const double dx[3], double dt);

/* EB level steps, MOL (oracle/_ref/libcamr_ref_eb.so only): the level
 * driver's step with the EB build's guards, the whole domain as one EB box.
 * Geometry over grow(domain, 5) as for orc_hydro_box_eb; state: valid
 * cells, updated in place (covered cells zero). */
long orc_eb_advance(const orc_params* p, const orc_level* lev, const unsigned* flag,
                    const double* vfrac, const double* ap0, const double* ap1, const double* ap2,
                    const double* fc0, const double* fc1, const double* fc2, const double* cent,
                    double* state, int nsteps, int first_step, double* dt_prev, double* dt_hist,
                    int redist);

/* initData's epilogue with the EB guards (rho > 0 only), valid cells. */
void orc_eb_init_finalize(const orc_params* p, const orc_level* lev, double* state);

/* clean_state on the valid cells (Source/CAMR.cpp:1253-1262). */
void orc_clean_state(const orc_params* p, const orc_level* lev, double* state);

#ifdef __cplusplus
}
#endif
#endif
