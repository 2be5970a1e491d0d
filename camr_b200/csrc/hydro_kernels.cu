#include "hydro_kernels.cuh"
#include "cell_point.cuh"

namespace camr {

namespace {

constexpr int kBlock = 128;

// Minimum resident blocks per SM of the heavy kernels (register budget):
// 4 for trace and flux3 (128 registers per thread) gave the shortest 256^3
// CTU-PPM step on B200 among 1/2/4; 6 for flux1 and flatten/divu (80
// registers, a few spills: 2.30 -> 2.04 and 1.36 -> 1.30 ms at 256^3);
// flux2 and the MOL fluxes keep their natural register count (the MOL
// fluxes measured no faster at 6).
#ifndef CAMR_MINB_TRACE
#define CAMR_MINB_TRACE 4
#endif
#ifndef CAMR_MINB_FLUX1
#define CAMR_MINB_FLUX1 6
#endif
#ifndef CAMR_MINB_FLUX2
#define CAMR_MINB_FLUX2 1
#endif
#ifndef CAMR_MINB_FLATDIVU
#define CAMR_MINB_FLATDIVU 6
#endif
#ifndef CAMR_MINB_MOLFLUX
#define CAMR_MINB_MOLFLUX 1
#endif
// Resident blocks asked of the MOL slope kernel (0: none).  Measured on
// B200 (256^3 MOL-PLM level): 8 (64 registers) 5.64 ms per step against
// 5.47 unbounded (72 registers); with the faces at 6 blocks (80 registers)
// as well, 5.86 + 12.75 against 5.47 + 12.17.
#ifndef CAMR_MINB_MOLSLOPE
#define CAMR_MINB_MOLSLOPE 0
#endif
#ifndef CAMR_MINB_FLUX3
#define CAMR_MINB_FLUX3 4
#endif
// 1: the level and per-box MOL paths run slopes and faces as one pass per
// direction (k_mol_fx / fy / fz).  Measured on B200 (256^3 MOL-PLM level):
// 22.5 ms for the fused faces against 6.5 + 13.6 ms for slopes + faces, so
// the default keeps the two kernels: the column walks of the y- and z-faces
// give each thread a long serial chain and fewer threads to hide it.
// 2: only the x-faces fused (row tiles), y and z as the two kernels: the
// fused x pass took 7.8 ms per step against about 6.6 ms for the x share of
// the two kernels (MOL level 28.2 against 26.7 ms), so the fusion loses
// even without the column walks.
#ifndef CAMR_MOLFUSE
#define CAMR_MOLFUSE 0
#endif
// 1: the MOL right-hand side runs as a cell pass and a face pass
// (k_mol_states + k_mol_face): each (cell, dir) turns its slopes into its
// two edge states at once, so the face pass reads two 9-slot records
// instead of both cells' primitive states and slopes.  0 (the default):
// slopes into HBM (k_mol_slope), then edge states + Riemann per face
// (k_mol_flux).  Measured on B200 (256^3 MOL-PLM level, ms per step):
// states 13.3 + faces 7.0 against slopes 6.5 + faces 13.6, so the edge-state
// arithmetic costs the same wherever it runs; batched two-level MOL step
// 129.7 ms (112.0 with 5 / 4 blocks per SM for the two batched stages)
// against 111.7, EB level 11.6 against 9.7 ms.  Bit-exact either way (the
// whole GPU suite passed with it on).  A workspace carved without the
// edge-state arrays (the adjoint's slope tape, the allocation-free entry
// point) always takes the slope path.
#ifndef CAMR_MOLSPLIT
#define CAMR_MOLSPLIT 0
#endif
#ifndef CAMR_MINB_MOLSTATES
#define CAMR_MINB_MOLSTATES 1
#endif
#ifndef CAMR_MINB_MOLFACE
#define CAMR_MINB_MOLFACE 1
#endif
// 1: the level and per-box CTU paths run the second and final flux passes
// as one kernel with the second-pass records in shared memory (k_flux23).
// Measured on B200 (256^3 CTU-PPM): 22.2 ms against 9.7 + 6.1 ms for the
// two kernels (two blocks of 8 warps per SM, a barrier per layer and a
// third, one-warp round of record work per layer), so the default keeps
// the two kernels and their records in HBM.
#ifndef CAMR_FLUX23
#define CAMR_FLUX23 0
#endif

inline unsigned grid_for(int64_t n) { return unsigned((n + kBlock - 1) / kBlock); }

__device__ __forceinline__ int64_t gtid() {
  return int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
}

__global__ void __launch_bounds__(kBlock) k_ctoprim(Region r, Space s, DFab u, DFab src,
                                                     bool has_src, KParams P, double* q,
                                                     double* srcq, DevError* err) {
  int i, j, k;
  if (!region_cell(r, gtid(), i, j, k)) return;
  ctoprim_body(i, j, k, s, u, src, has_src, P, q, srcq, err);
}

// ---------------------------------------------------------------------------
// K2: shock flattening of a cell (min over the three directions, as the
// reference's trace loops do: PLM Godunov_3D.cpp:109-115, PPM PPM.cpp:120-126)
// and the nodal divergence at the cell's low corner when it is a node of bx
// (Source/Hydro/Hydro_utils_K.H:12-169).
__device__ __forceinline__ void flatten_divu_body(int i, int j, int k, const Space& s,
                                                  const KGeom& g, const KParams& P,
                                                  bool do_flat, const double* q, double* flat,
                                                  double* divu) {
  const int64_t at = s.idx(i, j, k);
  if (do_flat) {
    double fl = 1.0;
    if (P.use_flattening == 1) {
      const int64_t st[3] = {1, s.sy, s.sz};
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        double pp[7], un[7];
#pragma unroll
        for (int o = -3; o <= 3; ++o) {
          pp[o + 3] = q[at + o * st[d] + SQ_P * s.sn];
          un[o + 3] = q[at + o * st[d] + (SQ_U + d) * s.sn];
        }
        fl = dmin(fl, flatten_dir(pp, un));
      }
    }
    flat[at] = fl;
  }
  if (i < g.lo[0] || j < g.lo[1] || k < g.lo[2] || i > g.hi[0] + 1 || j > g.hi[1] + 1 ||
      k > g.hi[2] + 1) {
    return;
  }
  const int NS = CAMR_BC_NOSLIPWALL;
  const double dxx = g.dx[0], dy = g.dx[1], dz = g.dx[2];
  auto Q = [&](int ii, int jj, int kk, int n) { return q[s.idx(ii, jj, kk) + n * s.sn]; };
  const int QUx = SQ_U, QVx = SQ_V, QWx = SQ_W;
  double ux = 0.25 * (Q(i, j, k, QUx) - Q(i - 1, j, k, QUx) + Q(i, j, k - 1, QUx) -
                      Q(i - 1, j, k - 1, QUx) + Q(i, j - 1, k, QUx) - Q(i - 1, j - 1, k, QUx) +
                      Q(i, j - 1, k - 1, QUx) - Q(i - 1, j - 1, k - 1, QUx)) / dxx;
  double vy = 0.25 * (Q(i, j, k, QVx) - Q(i, j - 1, k, QVx) + Q(i, j, k - 1, QVx) -
                      Q(i, j - 1, k - 1, QVx) + Q(i - 1, j, k, QVx) - Q(i - 1, j - 1, k, QVx) +
                      Q(i - 1, j, k - 1, QVx) - Q(i - 1, j - 1, k - 1, QVx)) / dy;
  double wz = 0.25 * (Q(i, j, k, QWx) - Q(i, j, k - 1, QWx) + Q(i - 1, j, k, QWx) -
                      Q(i - 1, j, k - 1, QWx) + Q(i, j - 1, k, QWx) - Q(i, j - 1, k - 1, QWx) +
                      Q(i - 1, j - 1, k, QWx) - Q(i - 1, j - 1, k - 1, QWx)) / dz;
  const int* dlo = g.dlo;
  const int* dhi = g.dhi;
  const int* bclo = g.bclo;
  const int* bchi = g.bchi;
  if (i == dlo[0] && bclo[0] == NS) {
    vy = 0.5 * (Q(i, j, k, QVx) - Q(i, j - 1, k, QVx) + Q(i, j, k - 1, QVx) - Q(i, j - 1, k - 1, QVx)) / dy;
    wz = 0.5 * (Q(i, j, k, QWx) - Q(i, j, k - 1, QWx) + Q(i, j - 1, k, QWx) - Q(i, j - 1, k - 1, QWx)) / dz;
  } else if (i == dhi[0] + 1 && bchi[0] == NS) {
    vy = 0.5 * (Q(i - 1, j, k, QVx) - Q(i - 1, j - 1, k, QVx) + Q(i - 1, j, k - 1, QVx) - Q(i - 1, j - 1, k - 1, QVx)) / dy;
    wz = 0.5 * (Q(i - 1, j, k, QWx) - Q(i - 1, j, k - 1, QWx) + Q(i - 1, j - 1, k, QWx) - Q(i - 1, j - 1, k - 1, QWx)) / dz;
  }
  if (j == dlo[1] && bclo[1] == NS) {
    ux = 0.5 * (Q(i, j, k, QUx) - Q(i - 1, j, k, QUx) + Q(i, j, k - 1, QUx) - Q(i - 1, j, k - 1, QUx)) / dxx;
    wz = 0.5 * (Q(i, j, k, QWx) - Q(i, j, k - 1, QWx) + Q(i - 1, j, k, QWx) - Q(i - 1, j, k - 1, QWx)) / dz;
  } else if (j == dhi[1] + 1 && bchi[1] == NS) {
    ux = 0.5 * (Q(i, j - 1, k, QUx) - Q(i - 1, j - 1, k, QUx) + Q(i, j - 1, k - 1, QUx) - Q(i - 1, j - 1, k - 1, QUx)) / dxx;
    wz = 0.5 * (Q(i, j - 1, k, QWx) - Q(i, j - 1, k - 1, QWx) + Q(i - 1, j - 1, k, QWx) - Q(i - 1, j - 1, k - 1, QWx)) / dz;
  }
  if (k == dlo[2] && bclo[2] == NS) {
    ux = 0.5 * (Q(i, j, k, QUx) - Q(i - 1, j, k, QUx) + Q(i, j - 1, k, QUx) - Q(i - 1, j - 1, k, QUx)) / dxx;
    vy = 0.5 * (Q(i, j, k, QVx) - Q(i, j - 1, k, QVx) + Q(i - 1, j, k, QVx) - Q(i - 1, j - 1, k, QVx)) / dy;
  } else if (k == dhi[2] + 1 && bchi[2] == NS) {
    ux = 0.5 * (Q(i, j, k - 1, QUx) - Q(i - 1, j, k - 1, QUx) + Q(i, j - 1, k - 1, QUx) - Q(i - 1, j - 1, k - 1, QUx)) / dxx;
    vy = 0.5 * (Q(i, j, k - 1, QVx) - Q(i, j - 1, k - 1, QVx) + Q(i - 1, j, k - 1, QVx) - Q(i - 1, j - 1, k - 1, QVx)) / dy;
  }
  if (j == dlo[1] && bclo[1] == NS && k == dlo[2] && bclo[2] == NS) {
    ux = (Q(i, j, k, QUx) - Q(i - 1, j, k, QUx)) / dxx;
  } else if ((j == dhi[1] + 1 && bchi[1] == NS) && (k == dlo[2] && bclo[2] == NS)) {
    ux = (Q(i, j - 1, k, QUx) - Q(i - 1, j - 1, k, QUx)) / dxx;
  } else if ((j == dlo[1] && bclo[1] == NS) && (k == dhi[2] + 1 && bchi[2] == NS)) {
    ux = (Q(i, j, k - 1, QUx) - Q(i - 1, j, k - 1, QUx)) / dxx;
  } else if ((j == dhi[1] + 1 && bchi[1] == NS) && (k == dhi[2] + 1 && bchi[2] == NS)) {
    ux = (Q(i, j - 1, k - 1, QUx) - Q(i - 1, j - 1, k - 1, QUx)) / dxx;
  }
  if (i == dlo[0] && bclo[0] == NS && k == dlo[2] && bclo[2] == NS) {
    vy = (Q(i, j, k, QVx) - Q(i, j - 1, k, QVx)) / dy;
  } else if ((i == dhi[0] + 1 && bchi[0] == NS) && (k == dlo[2] && bclo[2] == NS)) {
    vy = (Q(i - 1, j, k, QVx) - Q(i - 1, j - 1, k, QVx)) / dy;
  } else if ((i == dlo[0] && bclo[0] == NS) && (k == dhi[2] + 1 && bchi[2] == NS)) {
    vy = (Q(i, j, k - 1, QVx) - Q(i, j - 1, k - 1, QVx)) / dy;
  } else if ((i == dhi[0] + 1 && bchi[0] == NS) && (k == dhi[2] + 1 && bchi[2] == NS)) {
    vy = (Q(i - 1, j, k - 1, QVx) - Q(i - 1, j - 1, k - 1, QVx)) / dy;
  }
  if (i == dlo[0] && bclo[0] == NS && j == dlo[1] && bclo[1] == NS) {
    wz = (Q(i, j, k, QWx) - Q(i, j, k - 1, QWx)) / dz;
  } else if ((i == dhi[0] + 1 && bchi[0] == NS) && (j == dlo[1] && bclo[1] == NS)) {
    wz = (Q(i - 1, j, k, QWx) - Q(i - 1, j, k - 1, QWx)) / dz;
  } else if ((i == dlo[0] && bclo[0] == NS) && (j == dhi[1] + 1 && bchi[1] == NS)) {
    wz = (Q(i, j - 1, k, QWx) - Q(i, j - 1, k - 1, QWx)) / dz;
  } else if ((i == dhi[0] + 1 && bchi[0] == NS) && (j == dhi[1] + 1 && bchi[1] == NS)) {
    wz = (Q(i - 1, j - 1, k, QWx) - Q(i - 1, j - 1, k - 1, QWx)) / dz;
  }
  divu[at] = ux + vy + wz;
}

__global__ void __launch_bounds__(kBlock, CAMR_MINB_FLATDIVU) k_flatten_divu(Region r, Space s, KGeom g,
                                                          KParams P, bool do_flat,
                                                          const double* q, double* flat,
                                                          double* divu) {
  int i, j, k;
  if (!region_cell(r, gtid(), i, j, k)) return;
  flatten_divu_body(i, j, k, s, g, P, do_flat, q, flat, divu);
}

// ---------------------------------------------------------------------------
// K3: normal predictor of one cell in direction blockIdx.y: PPM with
// characteristic tracing (PPM.cpp:101-410) or PLM (Godunov_3D.cpp:104-152 +
// PLM.H:170-323).  Writes the plus state on the cell's low face (SP) and the
// minus state on its high face (SM).
template <int d>
__device__ __forceinline__ void trace_body(int i, int j, int k, const Space& s,
                                           const KGeom& g, const KParams& P,
                                           const DtRef& dtr, const double* q,
                                           const double* flat, double* smd, double* spd,
                                           const double* srcq = nullptr) {
  const int64_t at = s.idx(i, j, k);
  const int64_t st = (d == 0) ? 1 : (d == 1) ? s.sy : s.sz;
  const double dt = dtr.get();
  const double dtdx = dt / g.dx[d];
  const double fl = flat[at];
  constexpr int un_slot = SQ_U + d;
  constexpr int t1 = (d == 0) ? SQ_V : (d == 1) ? SQ_W : SQ_U;  // QUT of PPM.cpp:84-97
  constexpr int t2 = (d == 0) ? SQ_W : (d == 1) ? SQ_U : SQ_V;  // QUTT
  double qp_o[ES_N], qm_o[ES_N];

  auto stencil = [&](int slot, double* v) {
#pragma unroll
    for (int o = -2; o <= 2; ++o) v[o + 2] = q[at + o * st + slot * s.sn];
  };

  if (P.ppm_type == 1) {
    const double rho_c = q[at + SQ_RHO * s.sn];
    const double p_c = q[at + SQ_P * s.sn];
    const double cc = sqrt(P.gamma * p_c / rho_c);  // q_aux(QGAMC)*p/rho, PPM.cpp:113
    const double un = q[at + un_slot * s.sn];
    const double speeds[3] = {un - cc, un, un + cc};
    // rho, un, p, rhoe: all three waves of both integrals.
    Traced4 Ip, Im;
    const int slots4[4] = {SQ_RHO, un_slot, SQ_P, SQ_REINT};
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      double sv[5];
      stencil(slots4[v], sv);
      double smv, spv;
      ppm_reconstruct(sv[0], sv[1], sv[2], sv[3], sv[4], fl, smv, spv);
      const double s6 = 6.0 * sv[2] - 3.0 * (smv + spv);
      double* ipv = (v == 0) ? Ip.rho : (v == 1) ? Ip.un : (v == 2) ? Ip.p : Ip.re;
      double* imv = (v == 0) ? Im.rho : (v == 1) ? Im.un : (v == 2) ? Im.p : Im.re;
#pragma unroll
      for (int w = 0; w < 3; ++w) ppm_wave(smv, spv, s6, speeds[w], dtdx, ipv[w], imv[w]);
    }
    // Transverse velocities and species: only the u-wave integrals are read
    // (PPM.cpp:193-199, :303-305, :401-403).
    const int slots_mid[2 + NSPEC] = {t1, t2, SQ_FS, SQ_FS + 1, SQ_FS + 2};
    const int es_mid[2 + NSPEC] = {ES_U + (t1 - SQ_U), ES_U + (t2 - SQ_U), ES_FS, ES_FS + 1,
                                   ES_FS + 2};
#pragma unroll
    for (int v = 0; v < 2 + NSPEC; ++v) {
      double sv[5];
      stencil(slots_mid[v], sv);
      double smv, spv;
      ppm_reconstruct(sv[0], sv[1], sv[2], sv[3], sv[4], fl, smv, spv);
      const double s6 = 6.0 * sv[2] - 3.0 * (smv + spv);
      double ipm, imm;
      ppm_wave(smv, spv, s6, speeds[1], dtdx, ipm, imm);
      qp_o[es_mid[v]] = imm;
      qm_o[es_mid[v]] = ipm;
    }
    // The traced gamma (PPM.cpp:146-157) of a gamma-law gas: the stencil is
    // constant, so both edge values equal gamma exactly, the Colella-Sekora
    // limiter returns gamma and s6 = 0, hence every wave integral is gamma.
    const double gam_ref = P.gamma;
    double o_rho, o_un, o_p, o_re;
    ppm_project(Im, 0, gam_ref, un, cc, true, P, o_rho, o_un, o_p, o_re);
    qp_o[ES_RHO] = o_rho;
    qp_o[ES_U + d] = o_un;
    qp_o[ES_P] = o_p;
    qp_o[ES_REINT] = o_re;
    ppm_project(Ip, 2, gam_ref, un, cc, false, P, o_rho, o_un, o_p, o_re);
    qm_o[ES_RHO] = o_rho;
    qm_o[ES_U + d] = o_un;
    qm_o[ES_P] = o_p;
    qm_o[ES_REINT] = o_re;
  } else {
    // PLM: slopes of every traced component (PLM.H:19-79), then hydro_plm_d.
    double slope[ES_N];
    const int slot_of[ES_N] = {SQ_RHO, SQ_U, SQ_V, SQ_W, SQ_P, SQ_REINT, SQ_FS, SQ_FS + 1,
                               SQ_FS + 2};
#pragma unroll
    for (int n = 0; n < ES_N; ++n) {
      double sv[5];
      stencil(slot_of[n], sv);
      slope[n] = plm_slope(sv[0], sv[1], sv[2], sv[3], sv[4], fl, P.plm_iorder);
    }
    if (P.use_pslope) {
      // Godunov_3D.cpp:120-146: the pressure slope of plm_pslope, with
      // the primitive sources (zero when the box has none)
      double pv[5], rv[5], su[5];
      stencil(SQ_P, pv);
      stencil(SQ_RHO, rv);
#pragma unroll
      for (int o = 0; o < 5; ++o)
        su[o] = srcq ? srcq[at + (o - 2) * st + (ES_U + d) * s.sn] : 0.0;
      slope[ES_P] = plm_pslope(pv, rv, su, g.dx[d], fl, P.plm_iorder);
    }
    plm_edge_states<d>(q, at, s.sn, slope, dt / g.dx[d], P, qp_o, qm_o);
  }
  store_es(spd, s, at, qp_o);
  store_es(smd, s, at + st, qm_o);
}

__global__ void __launch_bounds__(kBlock, CAMR_MINB_TRACE) k_trace(Region r, Space s, KGeom g, KParams P,
                                                   DtRef dtr, const double* q,
                                                   const double* flat, double* sm0,
                                                   double* sm1, double* sm2, double* sp0,
                                                   double* sp1, double* sp2,
                                                   const double* srcq) {
  int i, j, k;
  if (!region_cell(r, gtid(), i, j, k)) return;
  switch (blockIdx.y) {
    case 0: trace_body<0>(i, j, k, s, g, P, dtr, q, flat, sm0, sp0, srcq); break;
    case 1: trace_body<1>(i, j, k, s, g, P, dtr, q, flat, sm1, sp1, srcq); break;
    default: trace_body<2>(i, j, k, s, g, P, dtr, q, flat, sm2, sp2, srcq); break;
  }
}

// ---------------------------------------------------------------------------
// K4: first-pass Riemann fluxes (Godunov_3D.cpp:180-216).  blockIdx.y = E.
template <int E>
__device__ __forceinline__ void flux1_body(int i, int j, int k, const Space& s, const KGeom& g,
                                           const KParams& P, const double* q, double* smE,
                                           double* spE, double* fE) {
  const int64_t st = (E == 0) ? 1 : (E == 1) ? s.sy : s.sz;
  const int64_t at = s.idx(i, j, k);
  double ql[ES_N], qr[ES_N], f[NVAR], qpres, qun;
  load_es(smE, s, at, ql);
  load_es(spE, s, at, qr);
  const CellAux aL = load_aux(q, s, at - st, P.gamma);
  const CellAux aR = load_aux(q, s, at, P.gamma);
  const int idx = (E == 0) ? i : (E == 1) ? j : k;
  cmpflx<E>(ql, qr, aL, aR, idx, g.bclo[E], g.bchi[E], g.dlo[E], g.dhi[E], P, f, qpres, qun);
  // The reference's first-pass cmpflx edits the predictor states in place at
  // a physical-boundary face; the transverse passes read the edited values.
  if (idx == g.dlo[E] || idx == g.dhi[E] + 1) {
    smE[at + ES_RHO * s.sn] = ql[ES_RHO];
    smE[at + ES_P * s.sn] = ql[ES_P];
    smE[at + ES_REINT * s.sn] = ql[ES_REINT];
    spE[at + ES_RHO * s.sn] = qr[ES_RHO];
    spE[at + ES_P * s.sn] = qr[ES_P];
    spE[at + ES_REINT * s.sn] = qr[ES_REINT];
  }
  fE[at + FR_RHO * s.sn] = f[URHO];
  fE[at + FR_MX * s.sn] = f[UMX];
  fE[at + FR_MY * s.sn] = f[UMY];
  fE[at + FR_MZ * s.sn] = f[UMZ];
  fE[at + FR_E * s.sn] = f[UEDEN];
#pragma unroll
  for (int sp = 0; sp < NSPEC; ++sp) fE[at + (FR_FS + sp) * s.sn] = f[UFS + sp];
  fE[at + FR_PRES * s.sn] = qpres;
  fE[at + FR_UN * s.sn] = qun;
}

__global__ void __launch_bounds__(kBlock, CAMR_MINB_FLUX1) k_flux1(Region r0, Region r1, Region r2, Space s,
                                                   KGeom g, KParams P, const double* q,
                                                   double* sm0, double* sm1, double* sm2,
                                                   double* sp0, double* sp1, double* sp2,
                                                   double* f0, double* f1, double* f2) {
  int i, j, k;
  switch (blockIdx.y) {
    case 0:
      if (region_cell(r0, gtid(), i, j, k)) flux1_body<0>(i, j, k, s, g, P, q, sm0, sp0, f0);
      break;
    case 1:
      if (region_cell(r1, gtid(), i, j, k)) flux1_body<1>(i, j, k, s, g, P, q, sm1, sp1, f1);
      break;
    default:
      if (region_cell(r2, gtid(), i, j, k)) flux1_body<2>(i, j, k, s, g, P, q, sm2, sp2, f2);
      break;
  }
}

struct Ptr6 {
  double* p[6];
};
struct Ptr3 {
  double* p[3];
};
struct Reg6 {
  Region r[6];
};

// ---------------------------------------------------------------------------
// K5: second pass "D|E": D-face states corrected by E fluxes (hydro_transdo,
// Godunov_3D.cpp:218-380), then the Riemann flux.  blockIdx.y = combo(D,E).
template <int D, int E>
__device__ __forceinline__ void flux2_record(int i, int j, int k, const Space& s, const KGeom& g,
                                             const KParams& P, const DtRef& dtr, const double* q,
                                             const double* smD, const double* spD,
                                             const double* fE, double* rec) {
  const int64_t stD = (D == 0) ? 1 : (D == 1) ? s.sy : s.sz;
  const int64_t stE = (E == 0) ? 1 : (E == 1) ? s.sy : s.sz;
  const int64_t at = s.idx(i, j, k);
  const double dt = dtr.get();
  const double cdtdx = 1.0 / 3.0 * dt / g.dx[E];
  double qm[ES_N], qp[ES_N], qn[ES_N];
  {
    // minus half of cell f - e_D
    const int64_t cell = at - stD;
    double lo[FR_N], hi[FR_N];
    load_fr(fE, s, cell, lo);
    load_fr(fE, s, cell + stE, hi);
    const TTerms t = transdo_terms(lo, hi, cdtdx);
    load_es(smD, s, at, qn);
    transdo_side(t, P.gamma, qn, cdtdx, P, qm);
  }
  {
    // plus half of cell f
    double lo[FR_N], hi[FR_N];
    load_fr(fE, s, at, lo);
    load_fr(fE, s, at + stE, hi);
    const TTerms t = transdo_terms(lo, hi, cdtdx);
    load_es(spD, s, at, qn);
    transdo_side(t, P.gamma, qn, cdtdx, P, qp);
  }
  const CellAux aL = load_aux(q, s, at - stD, P.gamma);
  const CellAux aR = load_aux(q, s, at, P.gamma);
  const int idx = (D == 0) ? i : (D == 1) ? j : k;
  double f[NVAR], qpres, qun;
  cmpflx<D>(qm, qp, aL, aR, idx, g.bclo[D], g.bchi[D], g.dlo[D], g.dhi[D], P, f, qpres, qun);
  rec[FR_RHO] = f[URHO];
  rec[FR_MX] = f[UMX];
  rec[FR_MY] = f[UMY];
  rec[FR_MZ] = f[UMZ];
  rec[FR_E] = f[UEDEN];
#pragma unroll
  for (int spc = 0; spc < NSPEC; ++spc) rec[FR_FS + spc] = f[UFS + spc];
  rec[FR_PRES] = qpres;
  rec[FR_UN] = qun;
}

template <int D, int E>
__device__ __forceinline__ void flux2_body(int i, int j, int k, const Space& s, const KGeom& g,
                                           const KParams& P, const DtRef& dtr, const double* q,
                                           const double* smD, const double* spD,
                                           const double* fE, double* o) {
  double rec[FR_N];
  flux2_record<D, E>(i, j, k, s, g, P, dtr, q, smD, spD, fE, rec);
  const int64_t at = s.idx(i, j, k);
#pragma unroll
  for (int n = 0; n < FR_N; ++n) o[at + n * s.sn] = rec[n];
}

__global__ void __launch_bounds__(kBlock, CAMR_MINB_FLUX2) k_flux2(Reg6 regs, Space s, KGeom g, KParams P,
                                                   DtRef dtr, const double* q, Ptr3 sm,
                                                   Ptr3 sp, Ptr3 f1, Ptr6 f2) {
  int i, j, k;
  const int64_t t = gtid();
#define CAMR_F2(D, E)                                                                   \
  case combo(D, E):                                                                     \
    if (region_cell(regs.r[combo(D, E)], t, i, j, k))                                   \
      flux2_body<D, E>(i, j, k, s, g, P, dtr, q, sm.p[D], sp.p[D], f1.p[E],             \
                       f2.p[combo(D, E)]);                                              \
    break;
  switch (blockIdx.y) {
    CAMR_F2(0, 1)
    CAMR_F2(0, 2)
    CAMR_F2(1, 0)
    CAMR_F2(1, 2)
    CAMR_F2(2, 0)
    CAMR_F2(2, 1)
    default: break;
  }
#undef CAMR_F2
}

// Artificial viscosity, species normalisation and area weighting of one
// face flux (Hydro_adjust_fluxes.cpp:13-44; hydro_artif_visc.H:7-64;
// Hydro_utils_K.H:207-234).  uL/uR: the conserved state of the cells left
// and right of the face; dv: divu at the face's 4 nodes (corner, +t1, +t2,
// +t1+t2).
template <int dir>
__device__ __forceinline__ void adjust_flux(double* f, const double* uL, const double* uR,
                                            const double* dv, int idx, double dx,
                                            const KGeom& g, const KParams& P, double area) {
  const double div = P.difmag * dmin(0.0, 0.25 * (dv[0] + dv[1] + dv[2] + dv[3]));
  const bool at_bndry = (idx == g.dlo[dir] && g.bclo[dir] == CAMR_BC_NOSLIPWALL) ||
                        (idx == g.dhi[dir] + 1 && g.bchi[dir] == CAMR_BC_NOSLIPWALL);
#pragma unroll
  for (int n = 0; n < NVAR; ++n) {
    if (n == UTEMP) continue;
    const bool is_tang_vel = (dir == 0 && (n == UMY || n == UMZ)) ||
                             (dir == 1 && (n == UMX || n == UMZ)) ||
                             (dir == 2 && (n == UMX || n == UMY));
    if (!(at_bndry && is_tang_vel)) f[n] += dx * div * (uR[n] - uL[n]);
  }
  f[UTEMP] = 0.0;
  double summ = 0.0;
#pragma unroll
  for (int n = UFS; n < UFS + NSPEC; ++n) summ += f[n];
  const double fac = (summ != 0.0) ? f[URHO] / summ : 1.0;
#pragma unroll
  for (int n = UFS; n < UFS + NSPEC; ++n) f[n] *= fac;
#pragma unroll
  for (int n = 0; n < NVAR; ++n) f[n] *= area;
}

template <int F, bool MET = false>
__device__ __forceinline__ void face_adjust_and_store(double* f, double qpres, double qun,
                                                      int i, int j, int k,
                                                      const Space& s, const KGeom& g,
                                                      const KParams& P, const DFab& uin,
                                                      const double* divu, DFab flx,
                                                      double* qf, const Metrics* M = nullptr) {
  constexpr int e0 = (F == 0), e1 = (F == 1), e2 = (F == 2);
  constexpr int t1 = (F == 0) ? 1 : 0;
  constexpr int t2 = (F == 2) ? 1 : 2;
  const int64_t st1 = (t1 == 0) ? 1 : (t1 == 1) ? s.sy : s.sz;
  const int64_t st2 = (t2 == 0) ? 1 : (t2 == 1) ? s.sy : s.sz;
  const int64_t at = s.idx(i, j, k);
  double dv[4];
  dv[0] = divu[at];
  dv[1] = divu[at + st1];
  dv[2] = divu[at + st2];
  dv[3] = divu[at + st1 + st2];
  double uL[NVAR], uR[NVAR];
#pragma unroll
  for (int n = 0; n < NVAR; ++n) {
    uL[n] = uin(i - e0, j - e1, k - e2, n);
    uR[n] = uin(i, j, k, n);
  }
  double area = (F == 0) ? g.dx[1] * g.dx[2] : (F == 1) ? g.dx[0] * g.dx[2]
                                                        : g.dx[0] * g.dx[1];
  // hydro_ext_flx (Hydro_utils_K.H:224-234) with the caller's face areas
  if constexpr (MET) area = M->a[F](i, j, k, 0);
  const int idx = (F == 0) ? i : (F == 1) ? j : k;
  adjust_flux<F>(f, uL, uR, dv, idx, g.dx[F], g, P, area);
#pragma unroll
  for (int n = 0; n < NVAR; ++n) flx(i, j, k, n) = f[n];
  qf[at] = qpres;
  qf[at + s.sn] = qun;
}

// ---------------------------------------------------------------------------
// K6: final fluxes on the F-faces of bx (Godunov_3D.cpp:388-452):
// hydro_transdd halves of the two cells, Riemann, then adjust_fluxes.
template <int F, bool MET = false>
__device__ __forceinline__ void flux3_body(int i, int j, int k, const Space& s, const KGeom& g,
                                           const KParams& P, const DtRef& dtr,
                                           const double* q, const double* srcq, bool has_src,
                                           const double* smF, const double* spF,
                                           const double* fa, const double* fb,
                                           const double* divu, const DFab& uin, DFab flx,
                                           double* qfF, const Metrics* M = nullptr) {
  constexpr int t0 = (F == 0) ? 1 : 0;
  constexpr int t1 = (F == 2) ? 1 : 2;
  const int64_t stF = (F == 0) ? 1 : (F == 1) ? s.sy : s.sz;
  const int64_t st0 = (t0 == 0) ? 1 : (t0 == 1) ? s.sy : s.sz;
  const int64_t st1 = (t1 == 0) ? 1 : (t1 == 1) ? s.sy : s.sz;
  const int64_t at = s.idx(i, j, k);
  const double dt = dtr.get();
  const double hdt = 0.5 * dt;
  const double cdtdx0 = 0.5 * dt / g.dx[t0];
  const double cdtdx1 = 0.5 * dt / g.dx[t1];
  double qm[ES_N], qp[ES_N], qn[ES_N], sq[ES_N];
#pragma unroll
  for (int n = 0; n < ES_N; ++n) sq[n] = 0.0;
  {
    const int64_t cell = at - stF;
    double a0[FR_N], a1[FR_N], b0[FR_N], b1[FR_N];
    load_fr(fa, s, cell, a0);
    load_fr(fa, s, cell + st0, a1);
    load_fr(fb, s, cell, b0);
    load_fr(fb, s, cell + st1, b1);
    const TDTerms t = transdd_terms(a0, a1, b0, b1, P.gamma, cdtdx0, cdtdx1);
    if (has_src) load_es(srcq, s, cell, sq);
    load_es(smF, s, at, qn);
    transdd_side(t, qn, sq, hdt, P, qm);
  }
  {
    double a0[FR_N], a1[FR_N], b0[FR_N], b1[FR_N];
    load_fr(fa, s, at, a0);
    load_fr(fa, s, at + st0, a1);
    load_fr(fb, s, at, b0);
    load_fr(fb, s, at + st1, b1);
    const TDTerms t = transdd_terms(a0, a1, b0, b1, P.gamma, cdtdx0, cdtdx1);
    if (has_src) load_es(srcq, s, at, sq);
    load_es(spF, s, at, qn);
    transdd_side(t, qn, sq, hdt, P, qp);
  }
  const CellAux aL = load_aux(q, s, at - stF, P.gamma);
  const CellAux aR = load_aux(q, s, at, P.gamma);
  const int idx = (F == 0) ? i : (F == 1) ? j : k;
  double f[NVAR], qpres, qun;
  cmpflx<F>(qm, qp, aL, aR, idx, g.bclo[F], g.bchi[F], g.dlo[F], g.dhi[F], P, f, qpres, qun);
  face_adjust_and_store<F, MET>(f, qpres, qun, i, j, k, s, g, P, uin, divu, flx, qfF, M);
}

template <bool MET>
__global__ void __launch_bounds__(kBlock, CAMR_MINB_FLUX3) k_flux3(Region r0, Region r1, Region r2, Space s,
                                                   KGeom g, KParams P, DtRef dtr,
                                                   const double* q, const double* srcq,
                                                   bool has_src, Ptr3 sm, Ptr3 sp, Ptr6 f2,
                                                   const double* divu, DFab uin, DFab fx,
                                                   DFab fy, DFab fz, Ptr3 qf, Metrics M) {
  int i, j, k;
  const int64_t t = gtid();
  switch (blockIdx.y) {
    case 0:
      if (region_cell(r0, t, i, j, k))
        flux3_body<0, MET>(i, j, k, s, g, P, dtr, q, srcq, has_src, sm.p[0], sp.p[0],
                           f2.p[combo(1, 2)], f2.p[combo(2, 1)], divu, uin, fx, qf.p[0], &M);
      break;
    case 1:
      if (region_cell(r1, t, i, j, k))
        flux3_body<1, MET>(i, j, k, s, g, P, dtr, q, srcq, has_src, sm.p[1], sp.p[1],
                           f2.p[combo(0, 2)], f2.p[combo(2, 0)], divu, uin, fy, qf.p[1], &M);
      break;
    default:
      if (region_cell(r2, t, i, j, k))
        flux3_body<2, MET>(i, j, k, s, g, P, dtr, q, srcq, has_src, sm.p[2], sp.p[2],
                           f2.p[combo(0, 1)], f2.p[combo(1, 0)], divu, uin, fz, qf.p[2], &M);
      break;
  }
}

// ---------------------------------------------------------------------------
// K5 + K6 fused (the level and per-box paths).  For the final fluxes on the
// F-faces, a block owns a column of kF23T0 x kF23T1 F-faces (transverse
// directions t0 < t1) and marches along F.  For each cell layer c it
// computes, into shared memory, the second-pass records that the final
// fluxes read -- (t0|t1) on the layer's t0-faces and (t1|t0) on its t1-faces
// (flux2_record: hydro_transdo halves + Riemann, Godunov_3D.cpp:218-380) --
// then the final fluxes of the F-faces between layers c-1 and c (flux3:
// hydro_transdd halves + Riemann + adjust_fluxes, :388-452).  Two layers of
// records stay in shared memory; none goes to HBM.  A record on the edge of
// a column is computed by both columns that read it (1/16 more records);
// the F range is cut into segments that start one layer early.
constexpr int kF23T0 = 16, kF23T1 = 16;
constexpr int kF23Threads = kF23T0 * kF23T1;
constexpr int kF23NA = (kF23T0 + 1) * kF23T1;  // (t0|t1) records of a layer
constexpr int kF23NB = kF23T0 * (kF23T1 + 1);  // (t1|t0) records of a layer
constexpr int kF23SmemCol = 2 * (kF23NA + kF23NB) * FR_N * int(sizeof(double));

template <int F>
__device__ __forceinline__ void flux23_column(const Space& s, const KGeom& g, const KParams& P,
                                              const DtRef& dtr, const double* q,
                                              const double* srcq, bool has_src, const Ptr3& sm,
                                              const Ptr3& sp, const Ptr3& f1,
                                              const double* divu, const DFab& uin,
                                              const DFab& flx, double* qfF, int seg_len,
                                              double* sh) {
  constexpr int t0 = (F == 0) ? 1 : 0;
  constexpr int t1 = (F == 2) ? 1 : 2;
  const int nt0 = g.hi[t0] - g.lo[t0] + 1;
  const int nt1 = g.hi[t1] - g.lo[t1] + 1;
  const int ncol0 = (nt0 + kF23T0 - 1) / kF23T0;
  const int ncol1 = (nt1 + kF23T1 - 1) / kF23T1;
  if (int(blockIdx.x) >= ncol0 * ncol1) return;
  const int p0base = g.lo[t0] + int(blockIdx.x % ncol0) * kF23T0;
  const int p1base = g.lo[t1] + int(blockIdx.x / ncol0) * kF23T1;
  const int f_begin = g.lo[F] + int(blockIdx.y) * seg_len;
  if (f_begin > g.hi[F] + 1) return;
  const int f_end = min(f_begin + seg_len - 1, g.hi[F] + 1);
  const double* smT0 = sm.p[t0];
  const double* spT0 = sp.p[t0];
  const double* smT1 = sm.p[t1];
  const double* spT1 = sp.p[t1];
  const double* f1T0 = f1.p[t0];
  const double* f1T1 = f1.p[t1];
  for (int c = f_begin - 1; c <= f_end; ++c) {
    const int L = (c - f_begin + 1) & 1;
    double* A = sh + L * (kF23NA + kF23NB) * FR_N;
    double* B = A + kF23NA * FR_N;
    for (int r = threadIdx.x; r < kF23NA + kF23NB; r += kF23Threads) {
      int idx[3];
      idx[F] = c;
      double rec[FR_N];
      if (r < kF23NA) {
        idx[t0] = p0base + r % (kF23T0 + 1);
        idx[t1] = p1base + r / (kF23T0 + 1);
        if (idx[t0] > g.hi[t0] + 1 || idx[t1] > g.hi[t1]) continue;
        flux2_record<t0, t1>(idx[0], idx[1], idx[2], s, g, P, dtr, q, smT0, spT0, f1T1, rec);
#pragma unroll
        for (int n = 0; n < FR_N; ++n) A[n * kF23NA + r] = rec[n];
      } else {
        const int rb = r - kF23NA;
        idx[t0] = p0base + rb % kF23T0;
        idx[t1] = p1base + rb / kF23T0;
        if (idx[t0] > g.hi[t0] || idx[t1] > g.hi[t1] + 1) continue;
        flux2_record<t1, t0>(idx[0], idx[1], idx[2], s, g, P, dtr, q, smT1, spT1, f1T0, rec);
#pragma unroll
        for (int n = 0; n < FR_N; ++n) B[n * kF23NB + rb] = rec[n];
      }
    }
    __syncthreads();
    if (c >= f_begin) {
      const int a0 = threadIdx.x % kF23T0, a1 = threadIdx.x / kF23T0;
      int idx[3];
      idx[F] = c;
      idx[t0] = p0base + a0;
      idx[t1] = p1base + a1;
      if (idx[t0] <= g.hi[t0] && idx[t1] <= g.hi[t1]) {
        const double* Am = sh + ((L ^ 1) * (kF23NA + kF23NB)) * FR_N;  // layer c - 1
        const double* Bm = Am + kF23NA * FR_N;
        const double* Ap = A;
        const double* Bp = B;
        const int ia = a1 * (kF23T0 + 1) + a0;  // t0-face low of the cell column
        const int ib = a1 * kF23T0 + a0;        // t1-face low
        const int i = idx[0], j = idx[1], k = idx[2];
        const int64_t stF = (F == 0) ? 1 : (F == 1) ? s.sy : s.sz;
        const int64_t at = s.idx(i, j, k);
        const double dt = dtr.get();
        const double hdt = 0.5 * dt;
        const double cdtdx0 = 0.5 * dt / g.dx[t0];
        const double cdtdx1 = 0.5 * dt / g.dx[t1];
        double qm[ES_N], qp[ES_N], qn[ES_N], sq[ES_N];
#pragma unroll
        for (int n = 0; n < ES_N; ++n) sq[n] = 0.0;
        {
          double a0r[FR_N], a1r[FR_N], b0r[FR_N], b1r[FR_N];
#pragma unroll
          for (int n = 0; n < FR_N; ++n) {
            a0r[n] = Am[n * kF23NA + ia];
            a1r[n] = Am[n * kF23NA + ia + 1];
            b0r[n] = Bm[n * kF23NB + ib];
            b1r[n] = Bm[n * kF23NB + ib + kF23T0];
          }
          const TDTerms t = transdd_terms(a0r, a1r, b0r, b1r, P.gamma, cdtdx0, cdtdx1);
          if (has_src) load_es(srcq, s, at - stF, sq);
          load_es(sm.p[F], s, at, qn);
          transdd_side(t, qn, sq, hdt, P, qm);
        }
        {
          double a0r[FR_N], a1r[FR_N], b0r[FR_N], b1r[FR_N];
#pragma unroll
          for (int n = 0; n < FR_N; ++n) {
            a0r[n] = Ap[n * kF23NA + ia];
            a1r[n] = Ap[n * kF23NA + ia + 1];
            b0r[n] = Bp[n * kF23NB + ib];
            b1r[n] = Bp[n * kF23NB + ib + kF23T0];
          }
          const TDTerms t = transdd_terms(a0r, a1r, b0r, b1r, P.gamma, cdtdx0, cdtdx1);
          if (has_src) load_es(srcq, s, at, sq);
          load_es(sp.p[F], s, at, qn);
          transdd_side(t, qn, sq, hdt, P, qp);
        }
        const CellAux aL = load_aux(q, s, at - stF, P.gamma);
        const CellAux aR = load_aux(q, s, at, P.gamma);
        const int fidx = (F == 0) ? i : (F == 1) ? j : k;
        double f[NVAR], qpres, qun;
        cmpflx<F>(qm, qp, aL, aR, fidx, g.bclo[F], g.bchi[F], g.dlo[F], g.dhi[F], P, f, qpres,
                  qun);
        face_adjust_and_store<F>(f, qpres, qun, i, j, k, s, g, P, uin, divu, flx, qfF);
      }
    }
    __syncthreads();
  }
}

// The x-faces (F = 0) with the same records, marching along z instead, so
// that consecutive threads stay consecutive in x: a block owns kF23T0
// x-faces x kF23T1 cells in y; per z-plane it computes the (1|2) records on
// the plane's y-faces and the (2|1) records on the z-faces above the plane
// (those below come from the previous plane), then the plane's x-faces.
constexpr int kF23XA = (kF23T0 + 1) * (kF23T1 + 1);  // (1|2) records of a plane
constexpr int kF23XB = (kF23T0 + 1) * kF23T1;        // (2|1) records of a z-face layer
constexpr int kF23SmemX = (kF23XA + 2 * kF23XB) * FR_N * int(sizeof(double));
constexpr int kF23Smem = (kF23SmemCol > kF23SmemX) ? kF23SmemCol : kF23SmemX;

__device__ __forceinline__ void flux23_x(const Space& s, const KGeom& g, const KParams& P,
                                         const DtRef& dtr, const double* q, const double* srcq,
                                         bool has_src, const Ptr3& sm, const Ptr3& sp,
                                         const Ptr3& f1, const double* divu, const DFab& uin,
                                         const DFab& flx, double* qf0, int seg_len, double* sh) {
  const int nfx = g.hi[0] - g.lo[0] + 2;  // x-faces
  const int ncx = (nfx + kF23T0 - 1) / kF23T0;
  const int ncy = (g.hi[1] - g.lo[1] + kF23T1) / kF23T1;
  if (int(blockIdx.x) >= ncx * ncy) return;
  const int i0 = g.lo[0] + int(blockIdx.x % ncx) * kF23T0;  // first x-face of the tile
  const int j0 = g.lo[1] + int(blockIdx.x / ncx) * kF23T1;
  const int k_begin = g.lo[2] + int(blockIdx.y) * seg_len;
  if (k_begin > g.hi[2]) return;
  const int k_end = min(k_begin + seg_len - 1, g.hi[2]);
  double* A = sh;                      // (1|2) on y-faces of the plane
  double* Bl[2] = {A + kF23XA * FR_N, A + kF23XA * FR_N + kF23XB * FR_N};
  // (2|1) records on the z-faces at k (layer (k - k_begin) & 1) and k + 1
  auto fill_b = [&](int kz, double* Bz) {
    for (int r = threadIdx.x; r < kF23XB; r += kF23Threads) {
      const int ci = i0 - 1 + r % (kF23T0 + 1);
      const int cj = j0 + r / (kF23T0 + 1);
      if (ci > g.hi[0] + 1 || cj > g.hi[1]) continue;
      double rec[FR_N];
      flux2_record<2, 1>(ci, cj, kz, s, g, P, dtr, q, sm.p[2], sp.p[2], f1.p[1], rec);
#pragma unroll
      for (int n = 0; n < FR_N; ++n) Bz[n * kF23XB + r] = rec[n];
    }
  };
  fill_b(k_begin, Bl[0]);
  for (int k = k_begin; k <= k_end; ++k) {
    const int L = (k - k_begin) & 1;
    double* Blo = Bl[L];
    double* Bhi = Bl[L ^ 1];
    for (int r = threadIdx.x; r < kF23XA + kF23XB; r += kF23Threads) {
      double rec[FR_N];
      if (r < kF23XA) {
        const int ci = i0 - 1 + r % (kF23T0 + 1);
        const int fj = j0 + r / (kF23T0 + 1);
        if (ci > g.hi[0] + 1 || fj > g.hi[1] + 1) continue;
        flux2_record<1, 2>(ci, fj, k, s, g, P, dtr, q, sm.p[1], sp.p[1], f1.p[2], rec);
#pragma unroll
        for (int n = 0; n < FR_N; ++n) A[n * kF23XA + r] = rec[n];
      } else {
        const int rb = r - kF23XA;
        const int ci = i0 - 1 + rb % (kF23T0 + 1);
        const int cj = j0 + rb / (kF23T0 + 1);
        if (ci > g.hi[0] + 1 || cj > g.hi[1]) continue;
        flux2_record<2, 1>(ci, cj, k + 1, s, g, P, dtr, q, sm.p[2], sp.p[2], f1.p[1], rec);
#pragma unroll
        for (int n = 0; n < FR_N; ++n) Bhi[n * kF23XB + rb] = rec[n];
      }
    }
    __syncthreads();
    const int a0 = threadIdx.x % kF23T0, a1 = threadIdx.x / kF23T0;
    const int i = i0 + a0, j = j0 + a1;
    if (i <= g.hi[0] + 1 && j <= g.hi[1]) {
      // records of the cells i-1 (tile x-cell a0) and i (a0 + 1)
      const int64_t at = s.idx(i, j, k);
      const double dt = dtr.get();
      const double hdt = 0.5 * dt;
      const double cdtdx0 = 0.5 * dt / g.dx[1];
      const double cdtdx1 = 0.5 * dt / g.dx[2];
      double qm[ES_N], qp[ES_N], qn[ES_N], sq[ES_N];
#pragma unroll
      for (int n = 0; n < ES_N; ++n) sq[n] = 0.0;
#pragma unroll
      for (int side = 0; side < 2; ++side) {
        const int xi = a0 + side;
        double a0r[FR_N], a1r[FR_N], b0r[FR_N], b1r[FR_N];
#pragma unroll
        for (int n = 0; n < FR_N; ++n) {
          a0r[n] = A[n * kF23XA + a1 * (kF23T0 + 1) + xi];
          a1r[n] = A[n * kF23XA + (a1 + 1) * (kF23T0 + 1) + xi];
          b0r[n] = Blo[n * kF23XB + a1 * (kF23T0 + 1) + xi];
          b1r[n] = Bhi[n * kF23XB + a1 * (kF23T0 + 1) + xi];
        }
        const TDTerms t = transdd_terms(a0r, a1r, b0r, b1r, P.gamma, cdtdx0, cdtdx1);
        if (side == 0) {
          if (has_src) load_es(srcq, s, at - 1, sq);
          load_es(sm.p[0], s, at, qn);
          transdd_side(t, qn, sq, hdt, P, qm);
        } else {
          if (has_src) load_es(srcq, s, at, sq);
          load_es(sp.p[0], s, at, qn);
          transdd_side(t, qn, sq, hdt, P, qp);
        }
      }
      const CellAux aL = load_aux(q, s, at - 1, P.gamma);
      const CellAux aR = load_aux(q, s, at, P.gamma);
      double f[NVAR], qpres, qun;
      cmpflx<0>(qm, qp, aL, aR, i, g.bclo[0], g.bchi[0], g.dlo[0], g.dhi[0], P, f, qpres, qun);
      face_adjust_and_store<0>(f, qpres, qun, i, j, k, s, g, P, uin, divu, flx, qf0);
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kF23Threads, 2) k_flux23(Space s, KGeom g, KParams P, DtRef dtr,
                                                          const double* q, const double* srcq,
                                                          bool has_src, Ptr3 sm, Ptr3 sp,
                                                          Ptr3 f1, const double* divu, DFab uin,
                                                          DFab fx, DFab fy, DFab fz, Ptr3 qf,
                                                          int seg_len) {
  extern __shared__ double sh[];
  switch (blockIdx.z) {
    case 0:
      flux23_x(s, g, P, dtr, q, srcq, has_src, sm, sp, f1, divu, uin, fx, qf.p[0], seg_len, sh);
      break;
    case 1:
      flux23_column<1>(s, g, P, dtr, q, srcq, has_src, sm, sp, f1, divu, uin, fy, qf.p[1],
                       seg_len, sh);
      break;
    default:
      flux23_column<2>(s, g, P, dtr, q, srcq, has_src, sm, sp, f1, divu, uin, fz, qf.p[2],
                       seg_len, sh);
      break;
  }
}

// ---------------------------------------------------------------------------
#if CAMR_MINB_MOLSLOPE > 0
#define CAMR_MOLSLOPE_BOUNDS __launch_bounds__(kBlock, CAMR_MINB_MOLSLOPE)
#else
#define CAMR_MOLSLOPE_BOUNDS __launch_bounds__(kBlock)
#endif
__global__ void CAMR_MOLSLOPE_BOUNDS k_mol_slope(Region r0, Region r1, Region r2, Space s,
                                                       KParams P, const double* q,
                                                       Ptr3 slope, int dbase) {
  int i, j, k;
  const int64_t t = gtid();
  switch (int(blockIdx.y) + dbase) {
    case 0:
      if (region_cell(r0, t, i, j, k)) mol_slope_body<0>(i, j, k, s, P, q, slope.p[0]);
      break;
    case 1:
      if (region_cell(r1, t, i, j, k)) mol_slope_body<1>(i, j, k, s, P, q, slope.p[1]);
      break;
    default:
      if (region_cell(r2, t, i, j, k)) mol_slope_body<2>(i, j, k, s, P, q, slope.p[2]);
      break;
  }
}

// MOL face pass: edge states + Riemann (mol_edges_cmpflx), then adjust_fluxes.
template <int d, bool MET = false>
__device__ __forceinline__ void mol_flux_body(int i, int j, int k, const Space& s,
                                              const KGeom& g, const KParams& P,
                                              const double* q, const double* sl,
                                              const double* divu, const DFab& uin, DFab flx,
                                              double* qfd, const Metrics* M = nullptr) {
  double f[NVAR], qpres, qun;
  mol_edges_cmpflx<d>(i, j, k, s, g, P, q, sl, f, qpres, qun);
  face_adjust_and_store<d, MET>(f, qpres, qun, i, j, k, s, g, P, uin, divu, flx, qfd, M);
}

template <bool MET>
__global__ void __launch_bounds__(kBlock, CAMR_MINB_MOLFLUX) k_mol_flux(Region r0, Region r1, Region r2, Space s,
                                                      KGeom g, KParams P, const double* q,
                                                      Ptr3 slope, const double* divu,
                                                      DFab uin, DFab fx, DFab fy, DFab fz,
                                                      Ptr3 qf, Metrics M, int dbase) {
  int i, j, k;
  const int64_t t = gtid();
  switch (int(blockIdx.y) + dbase) {
    case 0:
      if (region_cell(r0, t, i, j, k))
        mol_flux_body<0, MET>(i, j, k, s, g, P, q, slope.p[0], divu, uin, fx, qf.p[0], &M);
      break;
    case 1:
      if (region_cell(r1, t, i, j, k))
        mol_flux_body<1, MET>(i, j, k, s, g, P, q, slope.p[1], divu, uin, fy, qf.p[1], &M);
      break;
    default:
      if (region_cell(r2, t, i, j, k))
        mol_flux_body<2, MET>(i, j, k, s, g, P, q, slope.p[2], divu, uin, fz, qf.p[2], &M);
      break;
  }
}

// ---------------------------------------------------------------------------
// MOL as a cell pass and a face pass.  The cell pass stores, per direction
// d, the right state of the cell's low d-face (ES_* slots, complete) in
// rst[d] and the pieces of the left state of its high d-face (ML_* slots:
// the species stay unnormalised with their sum, because when the sum is
// below small_dens the reference takes the species of the cell on the
// other side, MOL_riemann_K.H:82-86) in lpc[d].  The face pass completes
// the left state, runs hydro_cmpflx and adjust_fluxes.  The operations and
// their order are those of mol_edges_cmpflx (mol_slope_compute,
// mol_cell_states, mol_face_from_states).
enum { ML_P = 0, ML_UN, ML_UT1, ML_UT2, ML_REINT, ML_FS, ML_SUM = ML_FS + NSPEC, ML_N };
static_assert(int(ML_N) <= int(ES_N), "left pieces fit an edge-state array");

template <int d>
__device__ __forceinline__ void mol_states_body(int i, int j, int k, const Space& s,
                                                const KParams& P, const double* q, double* lpc,
                                                double* rst) {
  const int64_t at = s.idx(i, j, k);
  const int64_t sn = s.sn;
  double sl[SL_N], qr[ES_N];
  MolLeft l;
  mol_slope_compute<d>(at, s, P, q, sl);
  mol_cell_states<d>(at, s, P, q, sl, qr, l);
  store_es(rst, s, at, qr);
  lpc[at + ML_P * sn] = l.p;
  lpc[at + ML_UN * sn] = l.un;
  lpc[at + ML_UT1 * sn] = l.ut1;
  lpc[at + ML_UT2 * sn] = l.ut2;
  lpc[at + ML_REINT * sn] = l.reint;
#pragma unroll
  for (int sp = 0; sp < NSPEC; ++sp) lpc[at + (ML_FS + sp) * sn] = l.spec[sp];
  lpc[at + ML_SUM * sn] = l.sum;
}

template <int d, bool MET = false>
__device__ __forceinline__ void mol_face_body(int i, int j, int k, const Space& s,
                                              const KGeom& g, const KParams& P,
                                              const double* q, const double* lpc,
                                              const double* rst, const double* divu,
                                              const DFab& uin, DFab flx, double* qfd,
                                              const Metrics* M = nullptr) {
  const int64_t st = (d == 0) ? 1 : (d == 1) ? s.sy : s.sz;
  const int64_t at = s.idx(i, j, k);
  const int64_t atL = at - st;
  const int64_t sn = s.sn;
  MolLeft l;
  l.p = ld_ro(lpc + atL + ML_P * sn);
  l.un = ld_ro(lpc + atL + ML_UN * sn);
  l.ut1 = ld_ro(lpc + atL + ML_UT1 * sn);
  l.ut2 = ld_ro(lpc + atL + ML_UT2 * sn);
  l.reint = ld_ro(lpc + atL + ML_REINT * sn);
#pragma unroll
  for (int sp = 0; sp < NSPEC; ++sp) l.spec[sp] = ld_ro(lpc + atL + (ML_FS + sp) * sn);
  l.sum = ld_ro(lpc + atL + ML_SUM * sn);
  l.c = ld_ro(q + atL + SQ_C * sn);
  l.csml = ld_ro(q + atL + SQ_CSML * sn);
  double qr[ES_N];
  load_es(rst, s, at, qr);
  const CellAux aR = load_aux(q, s, at, P.gamma);
  double f[NVAR], qpres, qun;
  mol_face_from_states<d>(i, j, k, s, g, P, q, l, qr, aR, f, qpres, qun);
  face_adjust_and_store<d, MET>(f, qpres, qun, i, j, k, s, g, P, uin, divu, flx, qfd, M);
}

__global__ void __launch_bounds__(kBlock, CAMR_MINB_MOLSTATES) k_mol_states(Region r0, Region r1, Region r2,
                                                                    Space s, KParams P,
                                                                    const double* q, Ptr3 lpc,
                                                                    Ptr3 rst) {
  int i, j, k;
  const int64_t t = gtid();
  switch (blockIdx.y) {
    case 0:
      if (region_cell(r0, t, i, j, k)) mol_states_body<0>(i, j, k, s, P, q, lpc.p[0], rst.p[0]);
      break;
    case 1:
      if (region_cell(r1, t, i, j, k)) mol_states_body<1>(i, j, k, s, P, q, lpc.p[1], rst.p[1]);
      break;
    default:
      if (region_cell(r2, t, i, j, k)) mol_states_body<2>(i, j, k, s, P, q, lpc.p[2], rst.p[2]);
      break;
  }
}

template <bool MET>
__global__ void __launch_bounds__(kBlock, CAMR_MINB_MOLFACE) k_mol_face(Region r0, Region r1, Region r2,
                                                                Space s, KGeom g, KParams P,
                                                                const double* q, Ptr3 lpc,
                                                                Ptr3 rst, const double* divu,
                                                                DFab uin, DFab fx, DFab fy,
                                                                DFab fz, Ptr3 qf, Metrics M) {
  int i, j, k;
  const int64_t t = gtid();
  switch (blockIdx.y) {
    case 0:
      if (region_cell(r0, t, i, j, k))
        mol_face_body<0, MET>(i, j, k, s, g, P, q, lpc.p[0], rst.p[0], divu, uin, fx, qf.p[0], &M);
      break;
    case 1:
      if (region_cell(r1, t, i, j, k))
        mol_face_body<1, MET>(i, j, k, s, g, P, q, lpc.p[1], rst.p[1], divu, uin, fy, qf.p[1], &M);
      break;
    default:
      if (region_cell(r2, t, i, j, k))
        mol_face_body<2, MET>(i, j, k, s, g, P, q, lpc.p[2], rst.p[2], divu, uin, fz, qf.p[2], &M);
      break;
  }
}

// ---------------------------------------------------------------------------
// MOL slopes and face pass fused (the level and per-box paths): a cell's
// slopes (mol_slope_compute) become its two edge states at once
// (mol_cell_states) and the face between two cells takes the left pieces of
// one and the right state of the other (mol_face_from_states); the slopes
// never go to HBM.  x-faces: a block covers kMolRow consecutive cells of an
// x-row and passes the left pieces to the next thread through shared
// memory.  y- and z-faces: each thread walks a column of cells along the
// face direction and carries the previous cell's left pieces in registers
// (segments of about 64 cells, each starting one cell early).
constexpr int kMolRow = 128;

__global__ void __launch_bounds__(kMolRow) k_mol_fx(Space s, KGeom g, KParams P, const double* q,
                                                    const double* divu, DFab uin, DFab fx,
                                                    double* qf0) {
  __shared__ MolLeft left[kMolRow];
  constexpr int per = kMolRow - 1;
  const int i = g.lo[0] + int(blockIdx.x) * per - 1 + int(threadIdx.x);
  const int j = g.lo[1] + int(blockIdx.y);
  const int k = g.lo[2] + int(blockIdx.z);
  const bool have = i <= g.hi[0] + 1;
  double qr[ES_N];
  MolLeft l;
  if (have) {
    const int64_t at = s.idx(i, j, k);
    double sl[SL_N];
    mol_slope_compute<0>(at, s, P, q, sl);
    mol_cell_states<0>(at, s, P, q, sl, qr, l);
    left[threadIdx.x] = l;
  }
  __syncthreads();
  if (have && threadIdx.x > 0) {
    CellAux aR;
    aR.c = l.c;
    aR.csml = l.csml;
    aR.gamc = P.gamma;
    double f[NVAR], qpres, qun;
    mol_face_from_states<0>(i, j, k, s, g, P, q, left[threadIdx.x - 1], qr, aR, f, qpres, qun);
    face_adjust_and_store<0>(f, qpres, qun, i, j, k, s, g, P, uin, divu, fx, qf0);
  }
}

template <int d>
__device__ __forceinline__ void mol_column(const Space& s, const KGeom& g, const KParams& P,
                                           const double* q, const double* divu,
                                           const DFab& uin, const DFab& flx, double* qfd,
                                           int seg) {
  constexpr int T = (d == 1) ? 2 : 1;  // the transverse direction besides x
  const int i = g.lo[0] + int(blockIdx.x) * kMolRow + int(threadIdx.x);
  if (i > g.hi[0]) return;
  const int t = g.lo[T] + int(blockIdx.y);
  const int f_begin = g.lo[d] + int(blockIdx.z) * seg;
  if (f_begin > g.hi[d] + 1) return;
  const int f_end = min(f_begin + seg - 1, g.hi[d] + 1);
  MolLeft prev;
  for (int c = f_begin - 1; c <= f_end; ++c) {
    int idx[3];
    idx[0] = i;
    idx[T] = t;
    idx[d] = c;
    const int64_t at = s.idx(idx[0], idx[1], idx[2]);
    double sl[SL_N], qr[ES_N];
    MolLeft l;
    mol_slope_compute<d>(at, s, P, q, sl);
    mol_cell_states<d>(at, s, P, q, sl, qr, l);
    if (c >= f_begin) {
      CellAux aR;
      aR.c = l.c;
      aR.csml = l.csml;
      aR.gamc = P.gamma;
      double f[NVAR], qpres, qun;
      mol_face_from_states<d>(idx[0], idx[1], idx[2], s, g, P, q, prev, qr, aR, f, qpres, qun);
      face_adjust_and_store<d>(f, qpres, qun, idx[0], idx[1], idx[2], s, g, P, uin, divu, flx,
                               qfd);
    }
    prev = l;
  }
}

__global__ void __launch_bounds__(kMolRow) k_mol_fy(Space s, KGeom g, KParams P, const double* q,
                                                    const double* divu, DFab uin, DFab fy,
                                                    double* qf1, int seg) {
  mol_column<1>(s, g, P, q, divu, uin, fy, qf1, seg);
}

__global__ void __launch_bounds__(kMolRow) k_mol_fz(Space s, KGeom g, KParams P, const double* q,
                                                    const double* divu, DFab uin, DFab fz,
                                                    double* qf2, int seg) {
  mol_column<2>(s, g, P, q, divu, uin, fz, qf2, seg);
}

// ---------------------------------------------------------------------------
// K7: hydro_consup (Hydro_utils_K.H:239-257) with pdivu (:175-202).
template <bool MET = false>
__device__ __forceinline__ void consup_body(int i, int j, int k, const Space& s, const KGeom& g,
                                            const DFab& fx, const DFab& fy, const DFab& fz,
                                            const Ptr3& qf, const DFab& dsdt,
                                            const Metrics* M = nullptr) {
  const int64_t at = s.idx(i, j, k);
  // face areas low/high in each direction and the cell volume
  double a0 = g.dx[1] * g.dx[2], a1 = g.dx[0] * g.dx[2], a2 = g.dx[0] * g.dx[1];
  double a0h = a0, a1h = a1, a2h = a2;
  double vol = g.dx[0] * g.dx[1] * g.dx[2];
  if constexpr (MET) {
    a0 = M->a[0](i, j, k, 0);
    a0h = M->a[0](i + 1, j, k, 0);
    a1 = M->a[1](i, j, k, 0);
    a1h = M->a[1](i, j + 1, k, 0);
    a2 = M->a[2](i, j, k, 0);
    a2h = M->a[2](i, j, k + 1, 0);
    vol = M->vol(i, j, k, 0);
  }
  const double* q1 = qf.p[0];
  const double* q2 = qf.p[1];
  const double* q3 = qf.p[2];
  const int64_t sn = s.sn;
  const double pdivu =
      0.5 *
      ((q1[at + 1] + q1[at]) * (q1[at + 1 + sn] * a0h - q1[at + sn] * a0) +
       (q2[at + s.sy] + q2[at]) * (q2[at + s.sy + sn] * a1h - q2[at + sn] * a1) +
       (q3[at + s.sz] + q3[at]) * (q3[at + s.sz + sn] * a2h - q3[at + sn] * a2)) /
      vol;
  const double volinv = 1.0 / vol;
#pragma unroll
  for (int n = 0; n < NVAR; ++n) {
    dsdt(i, j, k, n) += (fx(i, j, k, n) - fx(i + 1, j, k, n) + fy(i, j, k, n) -
                         fy(i, j + 1, k, n) + fz(i, j, k, n) - fz(i, j, k + 1, n)) *
                        volinv;
  }
  dsdt(i, j, k, UEINT) -= pdivu;
}

template <bool MET>
__global__ void __launch_bounds__(kBlock) k_consup(Region r, Space s, KGeom g, DFab fx,
                                                    DFab fy, DFab fz, Ptr3 qf, DFab dsdt,
                                                    Metrics M) {
  int i, j, k;
  if (!region_cell(r, gtid(), i, j, k)) return;
  consup_body<MET>(i, j, k, s, g, fx, fy, fz, qf, dsdt, &M);
}

// The caller's primitive state and qaux (QVAR / NQAUX comps, the reference's
// layout, Source/Utils/IndexDefines.H:54-77) and primitive sources into the
// hydro's own q record and edge-state-layout srcq, on grow(bx,4).
// QGAME / QTEMP / QGAMC / QDPDR / QDPDE are not read: the gamma-law EOS
// makes QGAMC = eos_gamma, which the kernels use directly.
__global__ void __launch_bounds__(kBlock) k_import_q(Region r, Space s, DFab qin, DFab qaux,
                                                      DFab srcqin, bool has_srcq, double* q,
                                                      double* srcq) {
  int i, j, k;
  if (!region_cell(r, gtid(), i, j, k)) return;
  const int64_t at = s.idx(i, j, k);
  q[at + SQ_RHO * s.sn] = qin(i, j, k, QRHO);
  q[at + SQ_U * s.sn] = qin(i, j, k, QU);
  q[at + SQ_V * s.sn] = qin(i, j, k, QV);
  q[at + SQ_W * s.sn] = qin(i, j, k, QW);
  q[at + SQ_P * s.sn] = qin(i, j, k, QPRES);
  q[at + SQ_REINT * s.sn] = qin(i, j, k, QREINT);
  for (int sp = 0; sp < NSPEC; ++sp) q[at + (SQ_FS + sp) * s.sn] = qin(i, j, k, QFS + sp);
  q[at + SQ_C * s.sn] = qaux(i, j, k, QC);
  q[at + SQ_CSML * s.sn] = qaux(i, j, k, QCSML);
  if (has_srcq) {
    srcq[at + ES_RHO * s.sn] = srcqin(i, j, k, QRHO);
    srcq[at + ES_U * s.sn] = srcqin(i, j, k, QU);
    srcq[at + ES_V * s.sn] = srcqin(i, j, k, QV);
    srcq[at + ES_W * s.sn] = srcqin(i, j, k, QW);
    srcq[at + ES_P * s.sn] = srcqin(i, j, k, QPRES);
    srcq[at + ES_REINT * s.sn] = srcqin(i, j, k, QREINT);
    for (int sp = 0; sp < NSPEC; ++sp) srcq[at + (ES_FS + sp) * s.sn] = srcqin(i, j, k, QFS + sp);
  }
}


// ---------------------------------------------------------------------------
// Batched (work-list) versions of the stages: one launch covers every box of
// a level.  Each work item is (box, sub-direction, region, first block); a
// block finds its item by binary search over the items' first-block prefix
// and runs the same per-cell body as the per-box kernels.  The grid may be
// smaller than the block count (persistent, grid-stride over blocks).

__device__ __forceinline__ int find_item(const BatchItem* items, int n, int64_t b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (items[mid].block0 <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <int STAGE>
__device__ __forceinline__ void batched_cell(const BoxCtx& c, int sub, int i, int j, int k,
                                             const KParams& P, const DtRef& dt, DevError* err) {
  const Work& w = c.w;
  if constexpr (STAGE == BS_CTOPRIM) {
    if (c.ebflag) {
      const int64_t f = (i - c.eblo[0]) +
                        int64_t(c.ebn[0]) * ((j - c.eblo[1]) + int64_t(c.ebn[1]) * (k - c.eblo[2]));
      if ((c.ebflag[f] & 3u) == 3u) {
        const int64_t at = w.s.idx(i, j, k);
        for (int n = 0; n < SQ_N; ++n) w.q[at + n * w.s.sn] = 0.;
        if (c.has_src)
          for (int n = 0; n < ES_N; ++n) w.srcq[at + n * w.s.sn] = 0.;
        return;
      }
    }
    ctoprim_body(i, j, k, w.s, c.uin, c.src, c.has_src, P, w.q, w.srcq, err);
  } else if constexpr (STAGE == BS_FLATDIVU) {
    flatten_divu_body(i, j, k, w.s, c.g, P, !c.mol, w.q, w.flat, w.divu);
  } else if constexpr (STAGE == BS_TRACE) {
    switch (sub) {
      case 0: trace_body<0>(i, j, k, w.s, c.g, P, dt, w.q, w.flat, w.sm[0], w.sp[0], w.srcq); break;
      case 1: trace_body<1>(i, j, k, w.s, c.g, P, dt, w.q, w.flat, w.sm[1], w.sp[1], w.srcq); break;
      default: trace_body<2>(i, j, k, w.s, c.g, P, dt, w.q, w.flat, w.sm[2], w.sp[2], w.srcq); break;
    }
  } else if constexpr (STAGE == BS_FLUX1) {
    switch (sub) {
      case 0: flux1_body<0>(i, j, k, w.s, c.g, P, w.q, w.sm[0], w.sp[0], w.f1[0]); break;
      case 1: flux1_body<1>(i, j, k, w.s, c.g, P, w.q, w.sm[1], w.sp[1], w.f1[1]); break;
      default: flux1_body<2>(i, j, k, w.s, c.g, P, w.q, w.sm[2], w.sp[2], w.f1[2]); break;
    }
  } else if constexpr (STAGE == BS_FLUX2) {
#define CAMR_BF2(D, E)                                                                  \
  case combo(D, E):                                                                     \
    flux2_body<D, E>(i, j, k, w.s, c.g, P, dt, w.q, w.sm[D], w.sp[D], w.f1[E],          \
                     w.f2[combo(D, E)]);                                                \
    break;
    switch (sub) {
      CAMR_BF2(0, 1)
      CAMR_BF2(0, 2)
      CAMR_BF2(1, 0)
      CAMR_BF2(1, 2)
      CAMR_BF2(2, 0)
      CAMR_BF2(2, 1)
      default: break;
    }
#undef CAMR_BF2
  } else if constexpr (STAGE == BS_FLUX3) {
    switch (sub) {
      case 0:
        flux3_body<0>(i, j, k, w.s, c.g, P, dt, w.q, w.srcq, c.has_src, w.sm[0], w.sp[0],
                      w.f2[combo(1, 2)], w.f2[combo(2, 1)], w.divu, c.uin, c.flx[0], w.qf[0]);
        break;
      case 1:
        flux3_body<1>(i, j, k, w.s, c.g, P, dt, w.q, w.srcq, c.has_src, w.sm[1], w.sp[1],
                      w.f2[combo(0, 2)], w.f2[combo(2, 0)], w.divu, c.uin, c.flx[1], w.qf[1]);
        break;
      default:
        flux3_body<2>(i, j, k, w.s, c.g, P, dt, w.q, w.srcq, c.has_src, w.sm[2], w.sp[2],
                      w.f2[combo(0, 1)], w.f2[combo(1, 0)], w.divu, c.uin, c.flx[2], w.qf[2]);
        break;
    }
  } else if constexpr (STAGE == BS_MOLSLOPE) {
    // the cell pass: slopes, or (split layout) the two edge states
#if CAMR_MOLSPLIT
    switch (sub) {
      case 0: mol_states_body<0>(i, j, k, w.s, P, w.q, w.sm[0], w.sp[0]); break;
      case 1: mol_states_body<1>(i, j, k, w.s, P, w.q, w.sm[1], w.sp[1]); break;
      default: mol_states_body<2>(i, j, k, w.s, P, w.q, w.sm[2], w.sp[2]); break;
    }
#else
    switch (sub) {
      case 0: mol_slope_body<0>(i, j, k, w.s, P, w.q, w.slope[0]); break;
      case 1: mol_slope_body<1>(i, j, k, w.s, P, w.q, w.slope[1]); break;
      default: mol_slope_body<2>(i, j, k, w.s, P, w.q, w.slope[2]); break;
    }
#endif
  } else if constexpr (STAGE == BS_MOLFLUX) {
#if CAMR_MOLSPLIT
    switch (sub) {
      case 0: mol_face_body<0>(i, j, k, w.s, c.g, P, w.q, w.sm[0], w.sp[0], w.divu, c.uin, c.flx[0], w.qf[0]); break;
      case 1: mol_face_body<1>(i, j, k, w.s, c.g, P, w.q, w.sm[1], w.sp[1], w.divu, c.uin, c.flx[1], w.qf[1]); break;
      default: mol_face_body<2>(i, j, k, w.s, c.g, P, w.q, w.sm[2], w.sp[2], w.divu, c.uin, c.flx[2], w.qf[2]); break;
    }
#else
    switch (sub) {
      case 0: mol_flux_body<0>(i, j, k, w.s, c.g, P, w.q, w.slope[0], w.divu, c.uin, c.flx[0], w.qf[0]); break;
      case 1: mol_flux_body<1>(i, j, k, w.s, c.g, P, w.q, w.slope[1], w.divu, c.uin, c.flx[1], w.qf[1]); break;
      default: mol_flux_body<2>(i, j, k, w.s, c.g, P, w.q, w.slope[2], w.divu, c.uin, c.flx[2], w.qf[2]); break;
    }
#endif
  } else {
    Ptr3 qf{{w.qf[0], w.qf[1], w.qf[2]}};
    consup_body(i, j, k, w.s, c.g, c.flx[0], c.flx[1], c.flx[2], qf, c.dsdt);
  }
}

// Stages (bit STAGE of the mask) whose blocks first copy their box context
// into shared memory: the compiler may then reload box-uniform values from
// there instead of holding them in registers or spilling them.  Measured
// per stage: ctoprim, flux1, flux2 and the MOL fluxes gain (two-level MOL
// step 90.3 -> 88.0 ms); flatten/divu, slopes and consup lose, and flux3
// spills more.
#ifndef CAMR_BOX_SMEM_MASK
#define CAMR_BOX_SMEM_MASK ((1 << BS_CTOPRIM) | (1 << BS_FLUX1) | (1 << BS_FLUX2) | (1 << BS_MOLFLUX))
#endif
static_assert(sizeof(BoxCtx) % 8 == 0, "box context copied as 8-byte words");

template <int STAGE, int MINB>
__global__ void __launch_bounds__(kBlock, MINB)
    kb_stage(const BoxCtx* __restrict__ boxes, const BatchItem* __restrict__ items, int nitems,
             const int* __restrict__ bitem, int64_t nblocks, int chunk, KParams P, DtRef dt,
             DevError* err) {
  constexpr bool kSmem = (CAMR_BOX_SMEM_MASK >> STAGE) & 1;
  __shared__ BoxCtx sbox[1];
  for (int64_t b = blockIdx.x; b < nblocks; b += gridDim.x) {
    const int it = bitem ? bitem[b] : find_item(items, nitems, b);
    const BatchItem item = items[it];
    if constexpr (kSmem) {
      __syncthreads();
      const unsigned long long* src =
          reinterpret_cast<const unsigned long long*>(boxes + item.box);
      unsigned long long* dst = reinterpret_cast<unsigned long long*>(sbox);
      for (int w = threadIdx.x; w < int(sizeof(BoxCtx) / 8); w += kBlock) dst[w] = src[w];
      __syncthreads();
    }
    const BoxCtx& c = kSmem ? sbox[0] : boxes[item.box];
    const int64_t base = (b - item.block0) * int64_t(kBlock) * chunk;
    for (int q = 0; q < chunk; ++q) {
      int i, j, k;
      if (region_cell(item.r, base + int64_t(q) * kBlock + threadIdx.x, i, j, k)) {
        batched_cell<STAGE>(c, item.sub, i, j, k, P, dt, err);
      }
    }
  }
}
}  // namespace

size_t work_doubles(const Space& s, bool mol, bool has_src, bool mol_split) {
  size_t c = SQ_N + 1 /*divu*/;
  if (has_src) c += ES_N;
  if (!mol) {
    c += 1 /*flat*/ + 6 * ES_N + 3 * FR_N + 6 * FR_N;
  } else if (mol_split && CAMR_MOLSPLIT) {
    c += 6 * ES_N;  // left pieces and right states per direction
  } else {
    c += 3 * SL_N;
  }
  c += 3 * 2 /*qf*/;
  return c * size_t(s.sn);
}

void work_carve(Work& w, double* base, bool mol, bool has_src, bool mol_split) {
  double* p = base;
  const int64_t sn = w.s.sn;
  auto take = [&](int ncomp) {
    double* r = p;
    p += int64_t(ncomp) * sn;
    return r;
  };
  w.q = take(SQ_N);
  w.divu = take(1);
  w.srcq = has_src ? take(ES_N) : nullptr;
  w.flat = nullptr;
  for (int d = 0; d < 3; ++d) w.sm[d] = w.sp[d] = w.f1[d] = w.slope[d] = nullptr;
  for (int c = 0; c < 6; ++c) w.f2[c] = nullptr;
  if (!mol) {
    w.flat = take(1);
    for (int d = 0; d < 3; ++d) {
      w.sm[d] = take(ES_N);
      w.sp[d] = take(ES_N);
      w.f1[d] = take(FR_N);
    }
    for (int c = 0; c < 6; ++c) w.f2[c] = take(FR_N);
  } else if (mol_split && CAMR_MOLSPLIT) {
    for (int d = 0; d < 3; ++d) {
      w.sm[d] = take(ES_N);  // ML_* left pieces of the cell's high face
      w.sp[d] = take(ES_N);  // right state of the cell's low face
    }
  } else {
    for (int d = 0; d < 3; ++d) w.slope[d] = take(SL_N);
  }
  for (int d = 0; d < 3; ++d) w.qf[d] = take(2);
}

cudaError_t launch_hydro_fluxes(const HydroLaunch& L, const Work& w, cudaStream_t st) {
  const KGeom& g = L.g;
  const Space& s = w.s;
  int lo4[3], hi4[3], lo1[3], hi1[3];
  for (int d = 0; d < 3; ++d) {
    lo4[d] = g.lo[d] - NGROW;
    hi4[d] = g.hi[d] + NGROW;
    lo1[d] = g.lo[d] - 1;
    hi1[d] = g.hi[d] + 1;
  }
  const Region r4 = make_region(lo4, hi4);
  const Region r1 = make_region(lo1, hi1);
  auto mark = [&](const char* what) {
    if (L.timer) L.timer->mark(st, what);
  };
  mark("ctoprim");
  if (L.ext_q) {
    k_import_q<<<grid_for(r4.count()), kBlock, 0, st>>>(r4, s, L.qin, L.qauxin, L.srcqin,
                                                         L.ext_srcq, w.q, w.srcq);
  } else {
    k_ctoprim<<<grid_for(r4.count()), kBlock, 0, st>>>(r4, s, L.uin, L.src, L.has_src, L.P, w.q,
                                                       w.srcq, L.err);
  }
  mark("flatten_divu");
  k_flatten_divu<<<grid_for(r1.count()), kBlock, 0, st>>>(r1, s, g, L.P, !L.mol, w.q, w.flat,
                                                          w.divu);
  count_launch(2);
  Ptr3 qf{{w.qf[0], w.qf[1], w.qf[2]}};
  if (!L.mol) {
    mark("trace");
    k_trace<<<dim3(grid_for(r1.count()), 3), kBlock, 0, st>>>(
        r1, s, g, L.P, L.dt, w.q, w.flat, w.sm[0], w.sm[1], w.sm[2], w.sp[0], w.sp[1], w.sp[2],
        w.srcq);
    // first pass: E-faces [lo,hi+1] x grow(bx,1) in the other directions
    Region rf[3];
    for (int E = 0; E < 3; ++E) {
      int lo[3], hi[3];
      for (int d = 0; d < 3; ++d) {
        lo[d] = (d == E) ? g.lo[d] : g.lo[d] - 1;
        hi[d] = (d == E) ? g.hi[d] + 1 : g.hi[d] + 1;
      }
      rf[E] = make_region(lo, hi);
    }
    int64_t m = 0;
    for (int E = 0; E < 3; ++E) m = (rf[E].count() > m) ? rf[E].count() : m;
    mark("flux1");
    k_flux1<<<dim3(grid_for(m), 3), kBlock, 0, st>>>(rf[0], rf[1], rf[2], s, g, L.P, w.q,
                                                    w.sm[0], w.sm[1], w.sm[2], w.sp[0],
                                                    w.sp[1], w.sp[2], w.f1[0], w.f1[1],
                                                    w.f1[2]);
    if (CAMR_FLUX23 && !L.M.on) {
      // second and final passes fused: the records of the second pass live
      // in shared memory only (k_flux23); caller metric arrays take the
      // two-kernel path below
      static bool attr_set = false;
      if (!attr_set) {
        cudaError_t ea = cudaFuncSetAttribute(k_flux23, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              kF23Smem);
        if (ea != cudaSuccess) return ea;
        attr_set = true;
      }
      int ncols = 0, nfaces = 0;
      for (int F = 1; F < 3; ++F) {
        const int t0 = 0, t1 = (F == 2) ? 1 : 2;
        const int c0 = (g.hi[t0] - g.lo[t0] + kF23T0) / kF23T0;
        const int c1 = (g.hi[t1] - g.lo[t1] + kF23T1) / kF23T1;
        ncols = std::max(ncols, c0 * c1);
        nfaces = std::max(nfaces, g.hi[F] - g.lo[F] + 2);
      }
      // the x-faces march along z over cell planes
      ncols = std::max(ncols, ((g.hi[0] - g.lo[0] + 2 + kF23T0 - 1) / kF23T0) *
                                  ((g.hi[1] - g.lo[1] + kF23T1) / kF23T1));
      nfaces = std::max(nfaces, g.hi[2] - g.lo[2] + 1);
      // segments of about 64 face layers (each recomputes one layer)
      const int nseg = std::max(1, (nfaces + 32) / 64);
      const int seg_len = (nfaces + nseg - 1) / nseg;
      Ptr3 sm{{w.sm[0], w.sm[1], w.sm[2]}}, sp{{w.sp[0], w.sp[1], w.sp[2]}},
          f1{{w.f1[0], w.f1[1], w.f1[2]}};
      mark("flux23");
      k_flux23<<<dim3(unsigned(ncols), unsigned(nseg), 3), kF23Threads, kF23Smem, st>>>(
          s, g, L.P, L.dt, w.q, w.srcq, L.has_src, sm, sp, f1, w.divu, L.uin, L.flx[0],
          L.flx[1], L.flx[2], qf, seg_len);
      count_launch(3);
    } else {
    // second pass "D|E": D-faces [lo,hi+1], F in grow 1, E in bx
    Reg6 r6;
    m = 0;
    for (int D = 0; D < 3; ++D)
      for (int E = 0; E < 3; ++E) {
        if (E == D) continue;
        const int F = 3 - D - E;
        int lo[3], hi[3];
        for (int d = 0; d < 3; ++d) {
          lo[d] = g.lo[d];
          hi[d] = g.hi[d];
        }
        hi[D] += 1;
        lo[F] -= 1;
        hi[F] += 1;
        r6.r[combo(D, E)] = make_region(lo, hi);
        m = (r6.r[combo(D, E)].count() > m) ? r6.r[combo(D, E)].count() : m;
      }
    Ptr3 sm{{w.sm[0], w.sm[1], w.sm[2]}}, sp{{w.sp[0], w.sp[1], w.sp[2]}},
        f1{{w.f1[0], w.f1[1], w.f1[2]}};
    Ptr6 f2;
    for (int c = 0; c < 6; ++c) f2.p[c] = w.f2[c];
    mark("flux2");
    k_flux2<<<dim3(grid_for(m), 6), kBlock, 0, st>>>(r6, s, g, L.P, L.dt, w.q, sm, sp, f1, f2);
    // final pass on the faces of bx
    Region rb[3];
    m = 0;
    for (int F = 0; F < 3; ++F) {
      int lo[3], hi[3];
      for (int d = 0; d < 3; ++d) {
        lo[d] = g.lo[d];
        hi[d] = g.hi[d];
      }
      hi[F] += 1;
      rb[F] = make_region(lo, hi);
      m = (rb[F].count() > m) ? rb[F].count() : m;
    }
    mark("flux3");
    if (L.M.on)
      k_flux3<true><<<dim3(grid_for(m), 3), kBlock, 0, st>>>(
          rb[0], rb[1], rb[2], s, g, L.P, L.dt, w.q, w.srcq, L.has_src, sm, sp, f2, w.divu, L.uin,
          L.flx[0], L.flx[1], L.flx[2], qf, L.M);
    else
      k_flux3<false><<<dim3(grid_for(m), 3), kBlock, 0, st>>>(
          rb[0], rb[1], rb[2], s, g, L.P, L.dt, w.q, w.srcq, L.has_src, sm, sp, f2, w.divu, L.uin,
          L.flx[0], L.flx[1], L.flx[2], qf, L.M);
    count_launch(4);
    }
  } else {
    Region rs[3], rb[3];
    int64_t ms = 0, mb = 0;
    for (int d = 0; d < 3; ++d) {
      int lo[3], hi[3], flo[3], fhi[3];
      for (int a = 0; a < 3; ++a) {
        lo[a] = flo[a] = g.lo[a];
        hi[a] = fhi[a] = g.hi[a];
      }
      lo[d] -= 1;
      hi[d] += 1;
      fhi[d] += 1;
      rs[d] = make_region(lo, hi);
      rb[d] = make_region(flo, fhi);
      ms = (rs[d].count() > ms) ? rs[d].count() : ms;
      mb = (rb[d].count() > mb) ? rb[d].count() : mb;
    }
    if (CAMR_MOLFUSE == 1 && !L.M.on && !L.keep_slopes) {
      // slopes, edge states and faces fused (k_mol_fx / fy / fz)
      const int nb[3] = {g.hi[0] - g.lo[0] + 1, g.hi[1] - g.lo[1] + 1, g.hi[2] - g.lo[2] + 1};
      mark("mol_faces");
      k_mol_fx<<<dim3(unsigned((nb[0] + 1 + kMolRow - 2) / (kMolRow - 1)), unsigned(nb[1]),
                      unsigned(nb[2])),
                 kMolRow, 0, st>>>(s, g, L.P, w.q, w.divu, L.uin, L.flx[0], qf.p[0]);
      const int segy = std::max(1, (nb[1] + 1 + 32) / 64), segz = std::max(1, (nb[2] + 1 + 32) / 64);
      const int leny = (nb[1] + 1 + segy - 1) / segy, lenz = (nb[2] + 1 + segz - 1) / segz;
      const unsigned gx = unsigned((nb[0] + kMolRow - 1) / kMolRow);
      k_mol_fy<<<dim3(gx, unsigned(nb[2]), unsigned(segy)), kMolRow, 0, st>>>(
          s, g, L.P, w.q, w.divu, L.uin, L.flx[1], qf.p[1], leny);
      k_mol_fz<<<dim3(gx, unsigned(nb[1]), unsigned(segz)), kMolRow, 0, st>>>(
          s, g, L.P, w.q, w.divu, L.uin, L.flx[2], qf.p[2], lenz);
      count_launch(3);
      return cudaGetLastError();
    }
    if (!w.slope[0]) {
      if (L.keep_slopes) return cudaErrorInvalidValue;  // a tape needs the slope layout
      Ptr3 lpc{{w.sm[0], w.sm[1], w.sm[2]}};
      Ptr3 rst{{w.sp[0], w.sp[1], w.sp[2]}};
      mark("mol_states");
      k_mol_states<<<dim3(grid_for(ms), 3), kBlock, 0, st>>>(rs[0], rs[1], rs[2], s, L.P, w.q,
                                                             lpc, rst);
      mark("mol_face");
      if (L.M.on)
        k_mol_face<true><<<dim3(grid_for(mb), 3), kBlock, 0, st>>>(
            rb[0], rb[1], rb[2], s, g, L.P, w.q, lpc, rst, w.divu, L.uin, L.flx[0], L.flx[1],
            L.flx[2], qf, L.M);
      else
        k_mol_face<false><<<dim3(grid_for(mb), 3), kBlock, 0, st>>>(
            rb[0], rb[1], rb[2], s, g, L.P, w.q, lpc, rst, w.divu, L.uin, L.flx[0], L.flx[1],
            L.flx[2], qf, L.M);
      count_launch(2);
      return cudaGetLastError();
    }
    int dbase = 0;
    if (CAMR_MOLFUSE == 2 && !L.M.on && !L.keep_slopes) {
      // x-faces fused by row tiles (k_mol_fx), y and z as two passes
      const int nx = g.hi[0] - g.lo[0] + 1;
      mark("mol_fx");
      k_mol_fx<<<dim3(unsigned((nx + 1 + kMolRow - 2) / (kMolRow - 1)), unsigned(g.hi[1] - g.lo[1] + 1),
                      unsigned(g.hi[2] - g.lo[2] + 1)),
                 kMolRow, 0, st>>>(s, g, L.P, w.q, w.divu, L.uin, L.flx[0], qf.p[0]);
      count_launch();
      dbase = 1;
    }
    Ptr3 sl{{w.slope[0], w.slope[1], w.slope[2]}};
    mark("mol_slope");
    k_mol_slope<<<dim3(grid_for(ms), 3 - dbase), kBlock, 0, st>>>(rs[0], rs[1], rs[2], s, L.P,
                                                                   w.q, sl, dbase);
    mark("mol_flux");
    if (L.M.on)
      k_mol_flux<true><<<dim3(grid_for(mb), 3 - dbase), kBlock, 0, st>>>(
          rb[0], rb[1], rb[2], s, g, L.P, w.q, sl, w.divu, L.uin, L.flx[0], L.flx[1], L.flx[2], qf,
          L.M, dbase);
    else
      k_mol_flux<false><<<dim3(grid_for(mb), 3 - dbase), kBlock, 0, st>>>(
          rb[0], rb[1], rb[2], s, g, L.P, w.q, sl, w.divu, L.uin, L.flx[0], L.flx[1], L.flx[2], qf,
          L.M, dbase);
    count_launch(2);
  }
  return cudaGetLastError();
}


// Resident blocks per SM asked of each batched stage.  A batched kernel
// reads its box's pointers, strides and geometry from the box table in
// global memory instead of the parameter space, and without a bound the
// compiler keeps them all in registers (MOL fluxes 142 registers against 90
// for the per-box kernel), which halves the resident warps.  With these
// bounds (a few spills of box-uniform values, served by L1) the two-level MOL
// step went from 98.7 to 90.2 ms and the batched CTU-PPM hydro of 350 boxes
// from 28.0 to 26.7 ms.
#ifndef CAMR_BMINB_CTOPRIM
#define CAMR_BMINB_CTOPRIM 8
#endif
#ifndef CAMR_BMINB_FLATDIVU
#define CAMR_BMINB_FLATDIVU 5
#endif
#ifndef CAMR_BMINB_TRACE
#define CAMR_BMINB_TRACE CAMR_MINB_TRACE
#endif
#ifndef CAMR_BMINB_FLUX1
#define CAMR_BMINB_FLUX1 5
#endif
#ifndef CAMR_BMINB_FLUX2
#define CAMR_BMINB_FLUX2 4
#endif
#ifndef CAMR_BMINB_FLUX3
#define CAMR_BMINB_FLUX3 CAMR_MINB_FLUX3
#endif
#ifndef CAMR_BMINB_MOLSLOPE
#define CAMR_BMINB_MOLSLOPE 8
#endif
#ifndef CAMR_BMINB_MOLFLUX
#define CAMR_BMINB_MOLFLUX 5
#endif
#ifndef CAMR_BMINB_CONSUP
#define CAMR_BMINB_CONSUP 8
#endif

int batched_min_blocks(int stage) {
  switch (stage) {
    case BS_CTOPRIM: return CAMR_BMINB_CTOPRIM;
    case BS_FLATDIVU: return CAMR_BMINB_FLATDIVU;
    case BS_TRACE: return CAMR_BMINB_TRACE;
    case BS_FLUX1: return CAMR_BMINB_FLUX1;
    case BS_FLUX2: return CAMR_BMINB_FLUX2;
    case BS_FLUX3: return CAMR_BMINB_FLUX3;
    case BS_MOLSLOPE: return CAMR_BMINB_MOLSLOPE;
    case BS_MOLFLUX: return CAMR_BMINB_MOLFLUX;
    default: return CAMR_BMINB_CONSUP;
  }
}

const void* batched_kernel(int stage) {
  switch (stage) {
    case BS_CTOPRIM: return reinterpret_cast<const void*>(&kb_stage<BS_CTOPRIM, CAMR_BMINB_CTOPRIM>);
    case BS_FLATDIVU: return reinterpret_cast<const void*>(&kb_stage<BS_FLATDIVU, CAMR_BMINB_FLATDIVU>);
    case BS_TRACE: return reinterpret_cast<const void*>(&kb_stage<BS_TRACE, CAMR_BMINB_TRACE>);
    case BS_FLUX1: return reinterpret_cast<const void*>(&kb_stage<BS_FLUX1, CAMR_BMINB_FLUX1>);
    case BS_FLUX2: return reinterpret_cast<const void*>(&kb_stage<BS_FLUX2, CAMR_BMINB_FLUX2>);
    case BS_FLUX3: return reinterpret_cast<const void*>(&kb_stage<BS_FLUX3, CAMR_BMINB_FLUX3>);
    case BS_MOLSLOPE: return reinterpret_cast<const void*>(&kb_stage<BS_MOLSLOPE, CAMR_BMINB_MOLSLOPE>);
    case BS_MOLFLUX: return reinterpret_cast<const void*>(&kb_stage<BS_MOLFLUX, CAMR_BMINB_MOLFLUX>);
    default: return reinterpret_cast<const void*>(&kb_stage<BS_CONSUP, CAMR_BMINB_CONSUP>);
  }
}

cudaError_t launch_batched_stage(int stage, const BoxCtx* boxes, const BatchItem* items,
                                 int nitems, const int* bitem, int64_t nblocks, int chunk,
                                 unsigned grid, const KParams& P, DtRef dt, DevError* err,
                                 cudaStream_t st) {
  if (nblocks <= 0) return cudaSuccess;
  if (grid == 0 || grid > nblocks) grid = unsigned(nblocks);
  switch (stage) {
#define CAMR_LB(S, M)                                                                     \
  case S:                                                                                 \
    kb_stage<S, M><<<grid, kBlock, 0, st>>>(boxes, items, nitems, bitem, nblocks, chunk, P, dt, \
                                            err);                                            \
    break;
    CAMR_LB(BS_CTOPRIM, CAMR_BMINB_CTOPRIM)
    CAMR_LB(BS_FLATDIVU, CAMR_BMINB_FLATDIVU)
    CAMR_LB(BS_TRACE, CAMR_BMINB_TRACE)
    CAMR_LB(BS_FLUX1, CAMR_BMINB_FLUX1)
    CAMR_LB(BS_FLUX2, CAMR_BMINB_FLUX2)
    CAMR_LB(BS_FLUX3, CAMR_BMINB_FLUX3)
    CAMR_LB(BS_MOLSLOPE, CAMR_BMINB_MOLSLOPE)
    CAMR_LB(BS_MOLFLUX, CAMR_BMINB_MOLFLUX)
    CAMR_LB(BS_CONSUP, CAMR_BMINB_CONSUP)
#undef CAMR_LB
    default: return cudaErrorInvalidValue;
  }
  count_launch();
  return cudaGetLastError();
}

// Regions of one box for each batched stage (the same ones the per-box
// launcher uses).  Returns the number of sub-regions written to out.
int stage_regions(int stage, const KGeom& g, Region* out) {
  int lo[3], hi[3];
  auto set = [&](int a_lo0, int a_lo1, int a_lo2, int a_hi0, int a_hi1, int a_hi2) {
    lo[0] = a_lo0; lo[1] = a_lo1; lo[2] = a_lo2;
    hi[0] = a_hi0; hi[1] = a_hi1; hi[2] = a_hi2;
  };
  switch (stage) {
    case BS_CTOPRIM:
      set(g.lo[0] - NGROW, g.lo[1] - NGROW, g.lo[2] - NGROW, g.hi[0] + NGROW, g.hi[1] + NGROW,
          g.hi[2] + NGROW);
      out[0] = make_region(lo, hi);
      return 1;
    case BS_FLATDIVU:
      set(g.lo[0] - 1, g.lo[1] - 1, g.lo[2] - 1, g.hi[0] + 1, g.hi[1] + 1, g.hi[2] + 1);
      out[0] = make_region(lo, hi);
      return 1;
    case BS_TRACE:
      set(g.lo[0] - 1, g.lo[1] - 1, g.lo[2] - 1, g.hi[0] + 1, g.hi[1] + 1, g.hi[2] + 1);
      for (int d = 0; d < 3; ++d) out[d] = make_region(lo, hi);
      return 3;
    case BS_FLUX1:
      for (int E = 0; E < 3; ++E) {
        for (int d = 0; d < 3; ++d) {
          lo[d] = (d == E) ? g.lo[d] : g.lo[d] - 1;
          hi[d] = g.hi[d] + 1;
        }
        out[E] = make_region(lo, hi);
      }
      return 3;
    case BS_FLUX2:
      for (int D = 0; D < 3; ++D)
        for (int E = 0; E < 3; ++E) {
          if (E == D) continue;
          const int F = 3 - D - E;
          for (int d = 0; d < 3; ++d) {
            lo[d] = g.lo[d];
            hi[d] = g.hi[d];
          }
          hi[D] += 1;
          lo[F] -= 1;
          hi[F] += 1;
          out[combo(D, E)] = make_region(lo, hi);
        }
      return 6;
    case BS_FLUX3:
    case BS_MOLFLUX:
      for (int F = 0; F < 3; ++F) {
        for (int d = 0; d < 3; ++d) {
          lo[d] = g.lo[d];
          hi[d] = g.hi[d];
        }
        hi[F] += 1;
        out[F] = make_region(lo, hi);
      }
      return 3;
    case BS_MOLSLOPE:
      for (int dd = 0; dd < 3; ++dd) {
        for (int d = 0; d < 3; ++d) {
          lo[d] = g.lo[d];
          hi[d] = g.hi[d];
        }
        lo[dd] -= 1;
        hi[dd] += 1;
        out[dd] = make_region(lo, hi);
      }
      return 3;
    default:
      set(g.lo[0], g.lo[1], g.lo[2], g.hi[0], g.hi[1], g.hi[2]);
      out[0] = make_region(lo, hi);
      return 1;
  }
}

cudaError_t launch_hydro(const HydroLaunch& L, const Work& w, cudaStream_t st) {
  cudaError_t e = launch_hydro_fluxes(L, w, st);
  if (e != cudaSuccess) return e;
  const Region rb = make_region(L.g.lo, L.g.hi);
  Ptr3 qf{{w.qf[0], w.qf[1], w.qf[2]}};
  if (L.M.on)
    k_consup<true><<<grid_for(rb.count()), kBlock, 0, st>>>(rb, w.s, L.g, L.flx[0], L.flx[1],
                                                            L.flx[2], qf, L.dsdt, L.M);
  else
    k_consup<false><<<grid_for(rb.count()), kBlock, 0, st>>>(rb, w.s, L.g, L.flx[0], L.flx[1],
                                                             L.flx[2], qf, L.dsdt, L.M);
  count_launch(1);
  return cudaGetLastError();
}

}  // namespace camr
