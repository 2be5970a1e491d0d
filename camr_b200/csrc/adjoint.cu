// Discrete adjoint of the MOL level step (SSP-RK2, PLM slopes, two-shock
// Riemann) on a periodic uniform level, with checkpoint-and-recompute over
// time steps.
//
// Forward: the single-level step of CAMR::CAMR_advance with do_mol = 1
// (Source/CAMR_advance.cpp:124-136) + post_timestep's clean_state, issued
// with the same kernels as camr_level_advance (so it gives the same bits);
// the dt of each step (computeInitialDt / computeNewDt) is recorded, and the
// state is kept every `checkpoint_every` steps.
//
// Backward, segment by segment from the last checkpoint: the segment's
// step-start states are recomputed from its checkpoint with the recorded
// dts, then each step is reversed:
//   S_old = clean(S_n); B = expand(S_old); k1 = L(B); S* = B + dt k1;
//   B2 = expand(S*); k2 = L(B2); S_{n+1} = clean^3(B2/2 + S_old/2 + dt/2 k2)
// read backwards, each L(.) through its vector-Jacobian product: the face
// flux VJP (edge states, Riemann, artificial viscosity, species
// normalisation), the p div u term, the MC-limited slopes, the nodal div u
// and ctoprim, and the periodic ghost fill folded back onto the valid cells.
// The dt sequence is frozen (no derivative through the CFL minimum).
// Contributions of one face or one slope to several cells are summed with
// FP64 atomics.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "adjoint_point.cuh"
#include "level_point.cuh"

namespace camr {
namespace {

using namespace adj;

static_assert(int(adj::QC) == int(SQ_C) && int(adj::QCS) == int(SQ_CSML) &&
                  int(adj::QY) == int(SQ_FS) && int(adj::QRE) == int(SQ_REINT),
              "primitive record slots");

struct APtr3 {
  double* p[3];
};

struct AdjGeom {
  LGeom L;   // the level's padded arrays
  Space sp;  // the hydro Space of the domain box
};

__device__ __forceinline__ Par par_of(const KParams& P) {
  Par r;
  r.gamma = P.gamma;
  r.small = P.small;
  r.small_dens = P.small_dens;
  r.small_pres = P.small_pres;
  r.smallu = P.smallu;
  r.small_num = P.small_num;
  r.difmag = P.difmag;
  r.eta1 = P.dual_energy_eta1;
  r.eta2 = P.dual_energy_eta2;
  r.small_temp = P.small_temp;
  r.dual_energy_update_E_from_e = P.dual_energy_update_E_from_e;
  return r;
}

__device__ __forceinline__ void atomic_add_cell(double* a, int64_t at, int64_t sn, const double* v,
                                                int n) {
  for (int c = 0; c < n; ++c)
    if (v[c] != 0.0) atomicAdd(a + at + c * sn, v[c]);
}

// Face VJP of direction d on the faces of the domain box: the face's share
// of the update (its flux in dSdt of the two cells and its interface p, u_n
// in their p div u), then face_vjp, scattered to the cells' primitive
// records, slopes, nodal div u and conserved states.
template <int d>
__device__ void adj_face_body(int i, int j, int k, const AdjGeom& G, const KParams& P,
                              const double* B, const double* q, const double* sl,
                              const double* divu, const double* qf, const double* Ldsdt,
                              double* Lq, double* Lsl, double* Ldivu, double* LB) {
  const LGeom& L = G.L;
  const Space& s = G.sp;
  const int64_t st = (d == 0) ? 1 : (d == 1) ? s.sy : s.sz;
  constexpr int t1 = (d == 0) ? 1 : 0;
  constexpr int t2 = (d == 2) ? 1 : 2;
  const int64_t st1 = (t1 == 0) ? 1 : (t1 == 1) ? s.sy : s.sz;
  const int64_t st2 = (t2 == 0) ? 1 : (t2 == 1) ? s.sy : s.sz;
  const int64_t atR = s.idx(i, j, k);
  const int64_t atL = atR - st;
  const int ci[3] = {i, j, k};
  const bool inR = ci[d] <= L.dhi[d];
  const bool inL = ci[d] - 1 >= L.dlo[d];
  const double vol = L.dx[0] * L.dx[1] * L.dx[2];
  const double volinv = 1.0 / vol;
  const double area = (d == 0) ? L.dx[1] * L.dx[2] : (d == 1) ? L.dx[0] * L.dx[2]
                                                            : L.dx[0] * L.dx[1];
  FaceOut bo;
  for (int n = 0; n < NV; ++n) {
    const double lr = inR ? Ldsdt[atR + n * s.sn] : 0.0;
    const double ll = inL ? Ldsdt[atL + n * s.sn] : 0.0;
    bo.f[n] = (lr - ll) * volinv;
  }
  // p div u: dSdt(c)[UEINT] -= 0.5 * sum_d (p_hi + p_lo) (u_hi a - u_lo a) / vol
  {
    const double* qp = qf;
    const double* qu = qf + s.sn;
    double bp = 0.0, bu = 0.0;
    const double h = 0.5 / vol;
    if (inR) {
      const double lp = -Ldsdt[atR + EINT * s.sn] * h;
      bp += lp * (qu[atR + st] * area - qu[atR] * area);
      bu += -lp * (qp[atR + st] + qp[atR]) * area;
    }
    if (inL) {
      const double lp = -Ldsdt[atL + EINT * s.sn] * h;
      bp += lp * (qu[atR] * area - qu[atL] * area);
      bu += lp * (qp[atR] + qp[atL]) * area;
    }
    bo.qpres = bp;
    bo.qun = bu;
  }
  FaceIn in, bin;
  for (int n = 0; n < NQ; ++n) {
    in.qL[n] = q[atL + n * s.sn];
    in.qR[n] = q[atR + n * s.sn];
    bin.qL[n] = 0.0;
    bin.qR[n] = 0.0;
  }
  for (int n = 0; n < NS; ++n) {
    in.sL[n] = sl[atL + n * s.sn];
    in.sR[n] = sl[atR + n * s.sn];
    bin.sL[n] = 0.0;
    bin.sR[n] = 0.0;
  }
  const int64_t nodes[4] = {atR, atR + st1, atR + st2, atR + st1 + st2};
  for (int c = 0; c < 4; ++c) {
    in.dv[c] = divu[nodes[c]];
    bin.dv[c] = 0.0;
  }
  const int64_t uR = L.idx(i, j, k);
  const int64_t uLat = uR - st;  // B shares the Space layout
  for (int n = 0; n < NV; ++n) {
    in.uL[n] = B[uLat + n * L.sn];
    in.uR[n] = B[uR + n * L.sn];
    bin.uL[n] = 0.0;
    bin.uR[n] = 0.0;
  }
  const Par Pr = par_of(P);
  FaceTape t;
  FaceOut fo;
  face_forward<d>(in, L.dx[d], area, Pr, t, fo);
  face_vjp<d>(in, L.dx[d], area, Pr, t, bo, bin);
  atomic_add_cell(Lq, atL, s.sn, bin.qL, NQ);
  atomic_add_cell(Lq, atR, s.sn, bin.qR, NQ);
  atomic_add_cell(Lsl, atL, s.sn, bin.sL, NS);
  atomic_add_cell(Lsl, atR, s.sn, bin.sR, NS);
  for (int c = 0; c < 4; ++c)
    if (bin.dv[c] != 0.0) atomicAdd(Ldivu + nodes[c], bin.dv[c]);
  atomic_add_cell(LB, uLat, L.sn, bin.uL, NV);
  atomic_add_cell(LB, uR, L.sn, bin.uR, NV);
}

// Face VJP launch shape: 128 threads; the minimum resident blocks per SM
// bounds the registers of this (register-heavy) kernel.
#ifndef CAMR_ADJ_FACE_MINB
#define CAMR_ADJ_FACE_MINB 2
#endif
constexpr int kFaceBlk = 128;

__global__ void __launch_bounds__(kFaceBlk, CAMR_ADJ_FACE_MINB) k_adj_face(Region r0, Region r1, Region r2, AdjGeom G,
                                                    KParams P, const double* B, const double* q,
                                                    APtr3 sl, const double* divu, APtr3 qf,
                                                    const double* Ldsdt, double* Lq, APtr3 Lsl,
                                                    double* Ldivu, double* LB) {
  int i, j, k;
  const int64_t t = tid();
  switch (blockIdx.y) {
    case 0:
      if (region_cell(r0, t, i, j, k))
        adj_face_body<0>(i, j, k, G, P, B, q, sl.p[0], divu, qf.p[0], Ldsdt, Lq, Lsl.p[0], Ldivu, LB);
      break;
    case 1:
      if (region_cell(r1, t, i, j, k))
        adj_face_body<1>(i, j, k, G, P, B, q, sl.p[1], divu, qf.p[1], Ldsdt, Lq, Lsl.p[1], Ldivu, LB);
      break;
    default:
      if (region_cell(r2, t, i, j, k))
        adj_face_body<2>(i, j, k, G, P, B, q, sl.p[2], divu, qf.p[2], Ldsdt, Lq, Lsl.p[2], Ldivu, LB);
      break;
  }
}

template <int d>
__device__ void adj_slope_body(int i, int j, int k, const Space& s, const KParams& P,
                               const double* q, const double* Lsl, double* Lq) {
  const int64_t at = s.idx(i, j, k);
  double bo[NS];
  bool any = false;
  for (int n = 0; n < NS; ++n) {
    bo[n] = Lsl[at + n * s.sn];
    any = any || bo[n] != 0.0;
  }
  if (!any || P.plm_iorder == 1) return;
  const int64_t st = (d == 0) ? 1 : (d == 1) ? s.sy : s.sz;
  double qm[NQ], q0[NQ], qp[NQ], bm[NQ], b0[NQ], bp[NQ];
  for (int n = 0; n < NQ; ++n) {
    qm[n] = q[at - st + n * s.sn];
    q0[n] = q[at + n * s.sn];
    qp[n] = q[at + st + n * s.sn];
    bm[n] = b0[n] = bp[n] = 0.0;
  }
  const Par Pr = par_of(P);
  SlopeTape t;
  double o[NS];
  slope_fwd<d>(qm, q0, qp, Pr, t, o);
  slope_vjp<d>(qm, q0, qp, Pr, t, bo, bm, b0, bp);
  atomic_add_cell(Lq, at - st, s.sn, bm, NQ);
  atomic_add_cell(Lq, at, s.sn, b0, NQ);
  atomic_add_cell(Lq, at + st, s.sn, bp, NQ);
}

// 128-thread blocks bounded to 3 per SM (168 registers, a few spills): at
// 156 registers a thread, 256-thread blocks left one block (8 warps) per SM.
constexpr int kSlopeBlk = 128;

__global__ void __launch_bounds__(kSlopeBlk, 3) k_adj_slope(Region r0, Region r1, Region r2, Space s,
                                                     KParams P, const double* q, APtr3 Lsl,
                                                     double* Lq) {
  int i, j, k;
  const int64_t t = tid();
  switch (blockIdx.y) {
    case 0:
      if (region_cell(r0, t, i, j, k)) adj_slope_body<0>(i, j, k, s, P, q, Lsl.p[0], Lq);
      break;
    case 1:
      if (region_cell(r1, t, i, j, k)) adj_slope_body<1>(i, j, k, s, P, q, Lsl.p[1], Lq);
      break;
    default:
      if (region_cell(r2, t, i, j, k)) adj_slope_body<2>(i, j, k, s, P, q, Lsl.p[2], Lq);
      break;
  }
}

// Nodal div u (Hydro_utils_K.H:12-169, interior nodes):
// ux = 0.25 * (sum over the 4 cells at x-index i of u - at i-1) / dx, etc.
__global__ void __launch_bounds__(kBlk) k_adj_divu(Region r, Space s, LGeom L,
                                                    const double* Ldivu, double* Lq) {
  int i, j, k;
  if (!region_cell(r, tid(), i, j, k)) return;
  const int64_t at = s.idx(i, j, k);
  const double b = Ldivu[at];
  if (b == 0.0) return;
  const double bx = b * 0.25 / L.dx[0], by = b * 0.25 / L.dx[1], bz = b * 0.25 / L.dx[2];
  for (int dk = -1; dk <= 0; ++dk)
    for (int dj = -1; dj <= 0; ++dj)
      for (int di = -1; di <= 0; ++di) {
        const int64_t c = s.idx(i + di, j + dj, k + dk);
        atomicAdd(Lq + c + adj::QU * s.sn, (di == 0) ? bx : -bx);
        atomicAdd(Lq + c + adj::QV * s.sn, (dj == 0) ? by : -by);
        atomicAdd(Lq + c + adj::QW * s.sn, (dk == 0) ? bz : -bz);
      }
}

// ctoprim VJP on the cells whose primitive record received adjoints.
__global__ void __launch_bounds__(kBlk) k_adj_ctoprim(Region r, Space s, KParams P,
                                                       const double* B, const double* Lq,
                                                       double* LB) {
  int i, j, k;
  if (!region_cell(r, tid(), i, j, k)) return;
  const int64_t at = s.idx(i, j, k);
  double bq[NQ];
  bool any = false;
  for (int n = 0; n < NQ; ++n) {
    bq[n] = Lq[at + n * s.sn];
    any = any || bq[n] != 0.0;
  }
  if (!any) return;
  double u[NV], bu[NV];
  for (int n = 0; n < NV; ++n) {
    u[n] = B[at + n * s.sn];
    bu[n] = 0.0;
  }
  ctoprim_vjp(u, par_of(P), bq, bu);
  for (int n = 0; n < NV; ++n) LB[at + n * s.sn] += bu[n];
}

// Adjoint of expand_state(S) (periodic FillPatch of cleaned values, then
// computeTemp) and of the clean before it: gather the adjoints of every
// copy of a valid cell (itself and its periodic images among the ghost
// cells), then the clean_state VJP at S.  out (valid cells) = or += result.
__global__ void __launch_bounds__(kBlk) k_adj_expand(LGeom L, KParams P, const double* S,
                                                      const double* LBp, double* out, int add) {
  int i, j, k;
  if (!valid_cell(L, tid(), i, j, k)) return;
  int n3[3];
  for (int d = 0; d < 3; ++d) n3[d] = L.dhi[d] - L.dlo[d] + 1;
  const int c[3] = {i, j, k};
  double acc[NV];
  for (int n = 0; n < NV; ++n) acc[n] = 0.0;
  for (int ok = -1; ok <= 1; ++ok)
    for (int oj = -1; oj <= 1; ++oj)
      for (int oi = -1; oi <= 1; ++oi) {
        const int o3[3] = {oi, oj, ok};
        int p3[3];
        bool inside = true;
        for (int d = 0; d < 3; ++d) {
          p3[d] = c[d] + o3[d] * n3[d];
          if (p3[d] < L.plo[d] || p3[d] >= L.plo[d] + L.pn[d]) inside = false;
        }
        if (!inside) continue;
        const int64_t at = L.idx(p3[0], p3[1], p3[2]);
        for (int n = 0; n < NV; ++n) acc[n] += LBp[at + n * L.sn];
      }
  double s[NV], b[NV];
  const int64_t at = L.idx(i, j, k);
  load_cell(S, L, at, s);
  for (int n = 0; n < NV; ++n) b[n] = 0.0;
  clean_vjp(s, par_of(P), acc, b);
  for (int n = 0; n < NV; ++n) {
    if (add) out[at + n * L.sn] += b[n];
    else out[at + n * L.sn] = b[n];
  }
}

// Adjoint of the end of the step: S_{n+1} = clean(clean(clean(S_pre))) (the
// second clean after the zero gravity source when add_grav_src), with
// S_pre = B2/2 + S_old/2 + dt/2 k2.  Writes the adjoints of B2 (valid
// cells; ghost cells zeroed by the caller), of S_old (first half) and of k2.
__global__ void __launch_bounds__(kBlk) k_adj_final(LGeom L, KParams P, const double* dtp,
                                                     const double* Spre, const double* Lout,
                                                     double* LB2, double* LSold,
                                                     double* Ldsdt) {
  int i, j, k;
  if (!valid_cell(L, tid(), i, j, k)) return;
  const double dt = *dtp;
  const int64_t at = L.idx(i, j, k);
  const Par Pr = par_of(P);
  const int ncl = P.add_grav_src ? 3 : 2;
  double st[3][NV];
  CleanTape tp;
  load_cell(Spre, L, at, st[0]);
  for (int c = 1; c < ncl; ++c) clean_fwd(st[c - 1], Pr, tp, st[c]);
  double lam[NV], lnext[NV];
  load_cell(Lout, L, at, lam);
  for (int c = ncl - 1; c >= 0; --c) {
    for (int n = 0; n < NV; ++n) lnext[n] = 0.0;
    clean_vjp(st[c], Pr, lam, lnext);
    for (int n = 0; n < NV; ++n) lam[n] = lnext[n];
  }
  for (int n = 0; n < NV; ++n) {
    LB2[at + n * L.sn] = 0.5 * lam[n];
    LSold[at + n * L.sn] = 0.5 * lam[n];
    Ldsdt[at + n * L.sn] = 0.5 * dt * lam[n];
  }
}

// Adjoint of S* = B + dt k1 given the adjoint of S*: LB (valid) = lam,
// Ldsdt = dt lam.
__global__ void __launch_bounds__(kBlk) k_adj_stage1(LGeom L, const double* dtp,
                                                      const double* Lstar, double* LB,
                                                      double* Ldsdt) {
  int i, j, k;
  if (!valid_cell(L, tid(), i, j, k)) return;
  const double dt = *dtp;
  const int64_t at = L.idx(i, j, k);
  for (int n = 0; n < NV; ++n) {
    const double v = Lstar[at + n * L.sn];
    LB[at + n * L.sn] = v;
    Ldsdt[at + n * L.sn] = dt * v;
  }
}

// Final adjoint of the step: lam_n = clean_vjp(S_n, LSold).
__global__ void __launch_bounds__(kBlk) k_adj_first_clean(LGeom L, KParams P, const double* Sn,
                                                           const double* LSold, double* lam) {
  int i, j, k;
  if (!valid_cell(L, tid(), i, j, k)) return;
  const int64_t at = L.idx(i, j, k);
  double s[NV], b[NV], out[NV];
  load_cell(Sn, L, at, s);
  load_cell(LSold, L, at, b);
  for (int n = 0; n < NV; ++n) out[n] = 0.0;
  clean_vjp(s, par_of(P), b, out);
  store_cell(lam, L, at, out);
}

// The state before the end-of-step cleans: S_pre = B2/2 + S_old/2 + dt/2 k2.
__global__ void __launch_bounds__(kBlk) k_store_pre(LGeom L, Space sp, const double* dtp,
                                                     const double* B2, const double* S_old,
                                                     FluxPtrs fp, double* out) {
  int i, j, k;
  if (!valid_cell(L, tid(), i, j, k)) return;
  const double dt = *dtp;
  const int64_t at = L.idx(i, j, k);
  double b[NV], so[NV], hs[NV];
  load_cell(B2, L, at, b);
  load_cell(S_old, L, at, so);
  cell_dsdt(L, sp, i, j, k, fp.f, fp.q, hs);
  for (int n = 0; n < NV; ++n) {
    double v = 0.5 * b[n] + 0.5 * so[n];
    v += 0.5 * dt * hs[n];
    out[at + n * L.sn] = v;
  }
}

// Forward intermediates of one step that its adjoint reads.
struct StepTape {
  double *Sn, *S_old, *B, *Sstar, *B2, *Spre;
  Work w1, w2;
};

}  // namespace
}  // namespace camr

using namespace camr;

struct camr_adjoint {
  KParams P;
  camr_hydro_params hp;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  AdjGeom G;
  int64_t ncell = 0;
  int every = 20;
  // forward arrays
  double *S = nullptr, *S_old = nullptr, *B = nullptr, *B2 = nullptr, *Sstar = nullptr;
  double* flx[3] = {nullptr, nullptr, nullptr};
  double *work1 = nullptr, *work2 = nullptr;
  Work w1, w2;
  double* dt_cur = nullptr;
  double* dt_hist = nullptr;
  int hist_cap = 0;
  unsigned long long* bits = nullptr;
  int* nstep = nullptr;
  DevError* err = nullptr;
  // adjoint arrays
  double *Lam = nullptr, *LB = nullptr, *LB2 = nullptr, *LSold = nullptr, *LStar = nullptr,
         *Ldsdt = nullptr, *Lq = nullptr, *Lsl = nullptr, *Ldivu = nullptr;
  // checkpoints (padded copies of S at steps 0, every, 2*every, ...) and the
  // step-start states of one segment
  std::vector<double*> ckpt;
  std::vector<double*> seg;
  // per-step tapes of one segment (kept when they fit in device memory)
  std::vector<double*> tape_mem;
  std::vector<StepTape> tapes;
  bool tapes_ok = false;
  double* Spre = nullptr;  // the S_pre of the recompute path
  int nsteps = 0;
  double* staging = nullptr;
  size_t sbytes = 0;
};

namespace {

unsigned nblk(int64_t n) { return unsigned((n + kBlk - 1) / kBlk); }

// One forward MOL step from a->S with dt read from *dtp, writing the step's
// intermediates into `t` (S_old, B, S*, B2, the two Works; S_pre when
// t.Spre is set; a copy of S_n when t.Sn is another array) and, when
// `advance`, the new state into a->S: the kernels of the level driver, in
// its order.  bits (may be NULL) receives the CFL minimum of the new state.
cudaError_t fwd_step_tape(camr_adjoint* a, const double* dtp, unsigned long long* bits,
                          const StepTape& t, bool advance) {
  cudaStream_t st = a->stream;
  const LGeom& L = a->G.L;
  const int64_t npad = int64_t(L.pn[0]) * L.pn[1] * L.pn[2];
  if (t.Sn && t.Sn != a->S) {
    cudaError_t e = cudaMemcpyAsync(t.Sn, a->S, a->sbytes, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
  }
  k_clean_copy<<<nblk(a->ncell), kBlk, 0, st>>>(L, a->P, a->S, t.S_old, a->err);
  k_expand<<<nblk(npad), kBlk, 0, st>>>(L, a->P, t.S_old, t.B, a->err);
  count_launch(2);
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
  H.P = a->P;
  H.has_src = false;
  H.mol = true;
  H.dt = DtRef{0.0, dtp};
  H.err = a->err;
  auto sdfab = [&](double* p) {
    DFab f;
    f.p = p;
    for (int d = 0; d < 3; ++d) f.lo[d] = L.plo[d];
    f.sy = L.sy;
    f.sz = L.sz;
    f.sn = L.sn;
    return f;
  };
  for (int d = 0; d < 3; ++d) H.flx[d] = sdfab(a->flx[d]);
  H.dsdt = sdfab(nullptr);
  H.uin = sdfab(t.B);
  H.src = H.uin;
  H.keep_slopes = true;  // the backward pass reads the forward slopes
  cudaError_t e = launch_hydro_fluxes(H, t.w1, st);
  if (e != cudaSuccess) return e;
  FluxPtrs fp1, fp2;
  for (int d = 0; d < 3; ++d) {
    fp1.f[d] = fp2.f[d] = a->flx[d];
    fp1.q[d] = t.w1.qf[d];
    fp2.q[d] = t.w2.qf[d];
  }
  k_update_mol1<<<nblk(a->ncell), kBlk, 0, st>>>(L, a->G.sp, a->P, dtp, t.B, t.S_old, fp1,
                                                 t.Sstar);
  k_expand<<<nblk(npad), kBlk, 0, st>>>(L, a->P, t.Sstar, t.B2, a->err);
  count_launch(2);
  H.uin = sdfab(t.B2);
  H.src = H.uin;
  e = launch_hydro_fluxes(H, t.w2, st);
  if (e != cudaSuccess) return e;
  if (t.Spre) {
    k_store_pre<<<nblk(a->ncell), kBlk, 0, st>>>(L, a->G.sp, dtp, t.B2, t.S_old, fp2, t.Spre);
    count_launch();
  }
  if (advance) {
    k_update_mol2<<<nblk(a->ncell), kBlk, 0, st>>>(L, a->G.sp, a->P, dtp, t.B2, t.S_old, fp2,
                                                   a->S, bits, a->err, 1);
    count_launch();
  }
  return cudaGetLastError();
}

StepTape scratch_tape(camr_adjoint* a) {
  StepTape t;
  t.Sn = a->S;
  t.S_old = a->S_old;
  t.B = a->B;
  t.Sstar = a->Sstar;
  t.B2 = a->B2;
  t.Spre = a->Spre;
  t.w1 = a->w1;
  t.w2 = a->w2;
  return t;
}

cudaError_t fwd_step(camr_adjoint* a, const double* dtp, unsigned long long* bits) {
  StepTape t = scratch_tape(a);
  t.Spre = nullptr;
  return fwd_step_tape(a, dtp, bits, t, true);
}

// Adjoint of one L(B) evaluation: Ldsdt (valid cells) -> LB (+=, padded).
cudaError_t hydro_adj(camr_adjoint* a, const double* Bp, const Work& w, double* LBp) {
  cudaStream_t st = a->stream;
  const LGeom& L = a->G.L;
  const Space& s = a->G.sp;
  const size_t lq_bytes = size_t(s.sn) * (NQ + 3 * NS + 1) * sizeof(double);
  cudaError_t e = cudaMemsetAsync(a->Lq, 0, lq_bytes, st);
  if (e != cudaSuccess) return e;
  APtr3 sl, qf, Lsl;
  for (int d = 0; d < 3; ++d) {
    sl.p[d] = w.slope[d];
    qf.p[d] = w.qf[d];
    Lsl.p[d] = a->Lsl + size_t(d) * NS * s.sn;
  }
  Region rf[3], rs[3];
  int64_t mf = 0, ms = 0;
  for (int F = 0; F < 3; ++F) {
    int lo[3], hi[3], lo2[3], hi2[3];
    for (int d = 0; d < 3; ++d) {
      lo[d] = lo2[d] = L.dlo[d];
      hi[d] = hi2[d] = L.dhi[d];
    }
    hi[F] += 1;
    lo2[F] -= 1;
    hi2[F] += 1;
    rf[F] = make_region(lo, hi);
    rs[F] = make_region(lo2, hi2);
    mf = std::max(mf, rf[F].count());
    ms = std::max(ms, rs[F].count());
  }
  k_adj_face<<<dim3(unsigned((mf + kFaceBlk - 1) / kFaceBlk), 3), kFaceBlk, 0, st>>>(
      rf[0], rf[1], rf[2], a->G, a->P, Bp, w.q, sl,
                                                 w.divu, qf, a->Ldsdt, a->Lq, Lsl, a->Ldivu,
                                                 LBp);
  k_adj_slope<<<dim3(unsigned((ms + kSlopeBlk - 1) / kSlopeBlk), 3), kSlopeBlk, 0, st>>>(
      rs[0], rs[1], rs[2], s, a->P, w.q, Lsl, a->Lq);
  int lo[3], hi[3];
  for (int d = 0; d < 3; ++d) {
    lo[d] = L.dlo[d];
    hi[d] = L.dhi[d] + 1;
  }
  const Region rn = make_region(lo, hi);
  k_adj_divu<<<nblk(rn.count()), kBlk, 0, st>>>(rn, s, L, a->Ldivu, a->Lq);
  for (int d = 0; d < 3; ++d) {
    lo[d] = L.dlo[d] - 2;
    hi[d] = L.dhi[d] + 2;
  }
  const Region rc = make_region(lo, hi);
  k_adj_ctoprim<<<nblk(rc.count()), kBlk, 0, st>>>(rc, s, a->P, Bp, a->Lq, LBp);
  count_launch(4);
  return cudaGetLastError();
}

// Reverse one step: a->Lam holds the adjoint of S_{n+1} (valid cells); `t`
// holds the step's forward intermediates.  On return a->Lam holds the
// adjoint of S_n.
cudaError_t adj_step(camr_adjoint* a, const double* dtp, const StepTape& t) {
  cudaStream_t st = a->stream;
  const LGeom& L = a->G.L;
  // padded adjoint arrays start from zero (ghost cells receive the scatter)
  const size_t b = a->sbytes;
  cudaError_t e = cudaMemsetAsync(a->LB2, 0, b, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(a->LB, 0, b, st);
  if (e != cudaSuccess) return e;
  k_adj_final<<<nblk(a->ncell), kBlk, 0, st>>>(L, a->P, dtp, t.Spre, a->Lam, a->LB2, a->LSold,
                                               a->Ldsdt);
  count_launch();
  e = hydro_adj(a, t.B2, t.w2, a->LB2);
  if (e != cudaSuccess) return e;
  k_adj_expand<<<nblk(a->ncell), kBlk, 0, st>>>(L, a->P, t.Sstar, a->LB2, a->LStar, 0);
  k_adj_stage1<<<nblk(a->ncell), kBlk, 0, st>>>(L, dtp, a->LStar, a->LB, a->Ldsdt);
  count_launch(2);
  e = hydro_adj(a, t.B, t.w1, a->LB);
  if (e != cudaSuccess) return e;
  k_adj_expand<<<nblk(a->ncell), kBlk, 0, st>>>(L, a->P, t.S_old, a->LB, a->LSold, 1);
  k_adj_first_clean<<<nblk(a->ncell), kBlk, 0, st>>>(L, a->P, t.Sn, a->LSold, a->Lam);
  count_launch(2);
  return cudaGetLastError();
}

// Per-step tapes for a segment of `every` steps, if they fit in half of the
// free device memory.
bool alloc_tapes(camr_adjoint* a) {
  if (a->tapes_ok) return true;
  const size_t wb = work_doubles(a->G.sp, true, false, false) * sizeof(double);
  const size_t per = 6 * a->sbytes + 2 * wb;
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return false;
  if (per * size_t(a->every) > free_b / 2) return false;
  for (int n = 0; n < a->every; ++n) {
    double* m = nullptr;
    if (cudaMalloc(reinterpret_cast<void**>(&m), per) != cudaSuccess) return false;
    a->tape_mem.push_back(m);
    StepTape t;
    double* p = m;
    auto take = [&](size_t bytes) {
      double* r = p;
      p += bytes / sizeof(double);
      return r;
    };
    t.Sn = take(a->sbytes);
    t.S_old = take(a->sbytes);
    t.B = take(a->sbytes);
    t.Sstar = take(a->sbytes);
    t.B2 = take(a->sbytes);
    t.Spre = take(a->sbytes);
    t.w1.s = t.w2.s = a->G.sp;
    work_carve(t.w1, take(wb), true, false, false);
    work_carve(t.w2, take(wb), true, false, false);
    a->tapes.push_back(t);
  }
  a->tapes_ok = true;
  return true;
}

void adj_free(camr_adjoint* a) {
  void* ptrs[] = {a->S, a->S_old, a->B, a->B2, a->Sstar, a->Spre, a->flx[0], a->flx[1], a->flx[2],
                  a->work1, a->work2, a->dt_cur, a->dt_hist, a->bits, a->nstep, a->err,
                  a->Lam, a->LB, a->LB2, a->LSold, a->LStar, a->Ldsdt, a->Lq, a->staging};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (double* p : a->ckpt) cudaFree(p);
  for (double* p : a->seg) cudaFree(p);
  for (double* p : a->tape_mem) cudaFree(p);
  if (a->own_stream) cudaStreamDestroy(a->stream);
  delete a;
}

}  // namespace

extern "C" {

camr_status camr_adjoint_create(const camr_geom* geom, const camr_hydro_params* p,
                                int checkpoint_every, void* stream, camr_adjoint** out) {
  if (!geom || !p || !out || checkpoint_every < 1) return CAMR_ERR_INVALID;
  if (!p->do_mol || p->riemann_solver != 0 || p->use_pslope) return CAMR_ERR_UNSUPPORTED;
  if (p->allow_small_energy != 1 || p->allow_negative_energy != 0) return CAMR_ERR_UNSUPPORTED;
  if (p->add_grav_src && p->const_grav != 0.0) return CAMR_ERR_UNSUPPORTED;
  for (int d = 0; d < 3; ++d)
    if (!geom->is_periodic[d] || geom->dom_hi[d] < geom->dom_lo[d]) return CAMR_ERR_UNSUPPORTED;
  camr_adjoint* a = new (std::nothrow) camr_adjoint();
  if (!a) return CAMR_ERR_NOMEM;
  a->hp = *p;
  a->P = make_kparams(*p);
  a->every = checkpoint_every;
  a->stream = static_cast<cudaStream_t>(stream);
  if (!a->stream) {
    if (cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete a;
      return CAMR_ERR_CUDA;
    }
    a->own_stream = true;
  }
  LGeom& L = a->G.L;
  for (int d = 0; d < 3; ++d) {
    L.dlo[d] = geom->dom_lo[d];
    L.dhi[d] = geom->dom_hi[d];
    L.plo[d] = geom->dom_lo[d] - NGROW;
    L.pn[d] = geom->dom_hi[d] - geom->dom_lo[d] + 1 + 2 * NGROW;
    L.periodic[d] = 1;
    L.bclo[d] = L.bchi[d] = 0;
    L.dx[d] = geom->dx[d];
    L.boxsz[d] = geom->dom_hi[d] - geom->dom_lo[d] + 1;
  }
  a->G.sp = make_space(L.dlo, L.dhi);
  L.sy = a->G.sp.sy;
  L.sz = a->G.sp.sz;
  L.sn = a->G.sp.sn;
  lgeom_finish(L);
  a->ncell = int64_t(L.dhi[0] - L.dlo[0] + 1) * (L.dhi[1] - L.dlo[1] + 1) *
             (L.dhi[2] - L.dlo[2] + 1);
  a->sbytes = size_t(L.sn) * NVAR * sizeof(double);
  a->hist_cap = 1 << 16;
  cudaError_t e = cudaSuccess;
  auto alloc = [&](double** ptr, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(ptr), bytes);
    if (e == cudaSuccess) e = cudaMemsetAsync(*ptr, 0, bytes, a->stream);
  };
  for (double** pp : {&a->S, &a->S_old, &a->B, &a->B2, &a->Sstar, &a->flx[0], &a->flx[1],
                      &a->flx[2], &a->Lam, &a->LB, &a->LB2, &a->LSold, &a->LStar, &a->Ldsdt,
                      &a->Spre})
    alloc(pp, a->sbytes);
  const size_t wb = work_doubles(a->G.sp, true, false, false) * sizeof(double);
  alloc(&a->work1, wb);
  alloc(&a->work2, wb);
  alloc(&a->Lq, size_t(L.sn) * (NQ + 3 * NS + 1) * sizeof(double));
  alloc(&a->dt_cur, sizeof(double));
  alloc(&a->dt_hist, sizeof(double) * a->hist_cap);
  alloc(&a->staging, size_t(a->ncell) * NVAR * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&a->bits), sizeof(*a->bits));
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&a->nstep), sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&a->err), sizeof(DevError));
  if (e == cudaSuccess) e = cudaMemsetAsync(a->err, 0, sizeof(DevError), a->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(a->stream);
  if (e != cudaSuccess) {
    adj_free(a);
    return CAMR_ERR_NOMEM;
  }
  a->Lsl = a->Lq + size_t(L.sn) * NQ;
  a->Ldivu = a->Lsl + size_t(L.sn) * 3 * NS;
  a->w1.s = a->w2.s = a->G.sp;
  work_carve(a->w1, a->work1, true, false, false);
  work_carve(a->w2, a->work2, true, false, false);
  *out = a;
  return CAMR_OK;
}

camr_status camr_adjoint_destroy(camr_adjoint* a) {
  if (!a) return CAMR_ERR_INVALID;
  adj_free(a);
  return CAMR_OK;
}

camr_status camr_adjoint_forward(camr_adjoint* a, const double* S0, double* S_final, int nsteps,
                                 const double* fixed_dts) {
  if (!a || !S0 || !S_final || nsteps < 1 || nsteps > a->hist_cap) return CAMR_ERR_INVALID;
  cudaStream_t st = a->stream;
  const LGeom& L = a->G.L;
  const size_t pk = size_t(a->ncell) * NVAR * sizeof(double);
  cudaError_t e = cudaMemcpyAsync(a->staging, S0, pk, cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess) return cuda_status_of(e);
  k_pack<<<nblk(a->ncell), kBlk, 0, st>>>(L, a->S, a->staging, 0);
  count_launch();
  if (fixed_dts) {
    e = cudaMemcpyAsync(a->dt_hist, fixed_dts, sizeof(double) * nsteps, cudaMemcpyHostToDevice,
                        st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_status_of(e);
  }
  // checkpoints: every `every` steps, padded copies
  const int nck = (nsteps + a->every - 1) / a->every;
  while (int(a->ckpt.size()) < nck) {
    double* p = nullptr;
    if (cudaMalloc(reinterpret_cast<void**>(&p), a->sbytes) != cudaSuccess) return CAMR_ERR_NOMEM;
    a->ckpt.push_back(p);
  }
  e = cudaMemsetAsync(a->nstep, 0, sizeof(int), st);
  if (e != cudaSuccess) return cuda_status_of(e);
  DtCtl c{a->hp.cfl, a->hp.max_dt, a->hp.fixed_dt, a->hp.initial_dt, a->hp.init_shrink,
          a->hp.change_max};
  for (int n = 0; n < nsteps; ++n) {
    if (n % a->every == 0) {
      e = cudaMemcpyAsync(a->ckpt[n / a->every], a->S, a->sbytes, cudaMemcpyDeviceToDevice, st);
      if (e != cudaSuccess) return cuda_status_of(e);
    }
    const double* dtp = a->dt_hist + n;
    if (!fixed_dts) {
      if (n == 0) {
        k_reset_bits<<<1, 1, 0, st>>>(a->bits);
        k_est_dt<<<nblk(a->ncell), kBlk, 0, st>>>(L, a->P, a->S, a->bits);
        count_launch(2);
      }
      k_dt_next<<<1, 1, 0, st>>>(c, n == 0 ? 1 : 0, nullptr, a->bits, a->dt_cur, a->dt_hist,
                                 a->nstep, a->hist_cap);
      count_launch();
    }
    e = fwd_step(a, dtp, fixed_dts ? nullptr : a->bits);
    if (e != cudaSuccess) return cuda_status_of(e);
  }
  a->nsteps = nsteps;
  k_pack<<<nblk(a->ncell), kBlk, 0, st>>>(L, a->S, a->staging, 1);
  count_launch();
  e = cudaMemcpyAsync(S_final, a->staging, pk, cudaMemcpyDeviceToDevice, st);
  return cuda_status_of(e);
}

camr_status camr_adjoint_backward(camr_adjoint* a, const double* lam_final, double* lam0) {
  if (!a || !lam_final || !lam0 || a->nsteps < 1) return CAMR_ERR_INVALID;
  cudaStream_t st = a->stream;
  const LGeom& L = a->G.L;
  const size_t pk = size_t(a->ncell) * NVAR * sizeof(double);
  cudaError_t e = cudaMemsetAsync(a->Lam, 0, a->sbytes, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(a->staging, lam_final, pk, cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess) return cuda_status_of(e);
  k_pack<<<nblk(a->ncell), kBlk, 0, st>>>(L, a->Lam, a->staging, 0);
  count_launch();
  while (int(a->seg.size()) < a->every) {
    double* p = nullptr;
    if (cudaMalloc(reinterpret_cast<void**>(&p), a->sbytes) != cudaSuccess) return CAMR_ERR_NOMEM;
    a->seg.push_back(p);
  }
  const int nseg = (a->nsteps + a->every - 1) / a->every;
  const bool taped = alloc_tapes(a);
  for (int sg = nseg - 1; sg >= 0; --sg) {
    const int n0 = sg * a->every;
    const int n1 = std::min(a->nsteps, n0 + a->every);
    e = cudaMemcpyAsync(a->S, a->ckpt[sg], a->sbytes, cudaMemcpyDeviceToDevice, st);
    if (taped) {
      // replay the segment keeping every step's intermediates
      for (int n = n0; n < n1 && e == cudaSuccess; ++n)
        e = fwd_step_tape(a, a->dt_hist + n, nullptr, a->tapes[n - n0], n + 1 < n1);
      for (int n = n1 - 1; n >= n0 && e == cudaSuccess; --n)
        e = adj_step(a, a->dt_hist + n, a->tapes[n - n0]);
    } else {
      // keep only the step-start states; recompute each step's intermediates
      for (int n = n0; n < n1 && e == cudaSuccess; ++n) {
        e = cudaMemcpyAsync(a->seg[n - n0], a->S, a->sbytes, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess && n + 1 < n1) e = fwd_step(a, a->dt_hist + n, nullptr);
      }
      const StepTape t = scratch_tape(a);
      for (int n = n1 - 1; n >= n0 && e == cudaSuccess; --n) {
        e = cudaMemcpyAsync(a->S, a->seg[n - n0], a->sbytes, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = fwd_step_tape(a, a->dt_hist + n, nullptr, t, false);
        if (e == cudaSuccess) e = adj_step(a, a->dt_hist + n, t);
      }
    }
    if (e != cudaSuccess) return cuda_status_of(e);
  }
  k_pack<<<nblk(a->ncell), kBlk, 0, st>>>(L, a->Lam, a->staging, 1);
  count_launch();
  e = cudaMemcpyAsync(lam0, a->staging, pk, cudaMemcpyDeviceToDevice, st);
  return cuda_status_of(e);
}

camr_status camr_adjoint_dts(camr_adjoint* a, double* dts, int n) {
  if (!a || !dts || n < 0 || n > a->nsteps) return CAMR_ERR_INVALID;
  cudaError_t e = cudaMemcpyAsync(dts, a->dt_hist, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                  a->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(a->stream);
  return cuda_status_of(e);
}

camr_status camr_adjoint_stream(camr_adjoint* a, void** stream) {
  if (!a || !stream) return CAMR_ERR_INVALID;
  *stream = static_cast<void*>(a->stream);
  return CAMR_OK;
}

camr_status camr_adjoint_get_error(camr_adjoint* a, camr_error_info* info) {
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
