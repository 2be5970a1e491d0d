// Embedded-boundary hydro of one box, MOL (SSP-RK2 right-hand side):
// hydro_umdrv_eb with do_mol = 1 (Source/Hydro/Hydro_umdrv_eb.cpp:14-191)
// and flux redistribution, as one stream of kernels:
//
//   K1 ctoprim            cells of grow(bx,5); covered cells get q = 0
//                         (CAMR_construct_hydro_source.cpp:101-111)
//   K2 EB slopes          cells of grow(bx,3), per direction; zero unless
//                         both neighbours are connected (MOL_hydro_eb_K.H)
//   K3 faces              faces of grow(bx,2), transverse +1: edge states +
//                         Riemann on connected faces, else zero
//                         (MOL/MOL_umeth_eb.cpp:21-191)
//   K4 EB div u           nodes of grow(bx,4) inside the (periodically grown)
//                         domain (Hydro_utils_eb_K.H:31-78); issued before K3
//   K5 adjust             artificial viscosity on every face of the flux
//                         box; species normalisation and area on open faces
//                         (Hydro_adjust_fluxes.cpp:48-171); inside K3's
//                         kernel, after each face's flux
//   K6 divergence         cells of grow(bx,2): face-centroid interpolated
//                         fluxes, the wall flux of cut cells, -div, p div u,
//                         the redistribution weight (Hydro_consup.cpp:29-98,
//                         Hydro_utils_eb_K.H:82-575, Hydro_hypflux_eb_K.H)
//   K7/K8 redistribution  flux redistribution (restated AMReX FluxRedist):
//                         per cut cell of grow(bx,1) the neighbourhood
//                         average and the mass to move, then each cell of bx
//                         gathers what its cut neighbours send, in raster
//                         order of the senders.
//
// Geometry (flags, volume and area fractions, face centroids) comes from
// the caller over a region G covering grow(bx,5).
//
// The EB level (camr_eb_level_*) runs the single-level MOL step around
// these kernels with the EB build's covered-cell guards, on the domain as
// one box with a persistent workspace.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstring>
#include <new>
#include <vector>

#include "cell_point.cuh"
#include "hydro_kernels.cuh"
#include "level_point.cuh"

namespace camr {
namespace {

constexpr int kEB = 128;

__device__ __forceinline__ int64_t etid() { return int64_t(blockIdx.x) * blockDim.x + threadIdx.x; }
inline unsigned eblk(int64_t n) { return unsigned((n + kEB - 1) / kEB); }

__device__ __forceinline__ bool f_covered(unsigned w) { return (w & 3u) == 3u; }
__device__ __forceinline__ bool f_regular(unsigned w) { return (w & 3u) == 0u; }
__device__ __forceinline__ bool f_single(unsigned w) { return (w & 3u) == 1u; }
__device__ __forceinline__ bool f_conn(unsigned w, int di, int dj, int dk) {
  return (w >> (2 + (di + 1) + 3 * (dj + 1) + 9 * (dk + 1))) & 1u;
}

// Geometry views over G (cells) and surroundingNodes(G, d) (faces).
struct EBG {
  const unsigned* flag;
  const double* vfrac;
  const double* ap[3];
  const double* fc[3];
  const double* cent;  // 3 comps of cell-centroid offsets, or null (cell centres)
  int lo[3], n[3];
  __device__ __forceinline__ int64_t c(int i, int j, int k) const {
    return (i - lo[0]) + int64_t(n[0]) * ((j - lo[1]) + int64_t(n[1]) * (k - lo[2]));
  }
  __device__ __forceinline__ int64_t f(int d, int i, int j, int k) const {
    const int nx = n[0] + (d == 0), ny = n[1] + (d == 1);
    return (i - lo[0]) + int64_t(nx) * ((j - lo[1]) + int64_t(ny) * (k - lo[2]));
  }
  __device__ __forceinline__ int64_t fn(int d) const {
    return int64_t(n[0] + (d == 0)) * (n[1] + (d == 1)) * (n[2] + (d == 2));
  }
  __device__ __forceinline__ unsigned fl(int i, int j, int k) const { return flag[c(i, j, k)]; }
  __device__ __forceinline__ double vf(int i, int j, int k) const { return vfrac[c(i, j, k)]; }
  __device__ __forceinline__ double ce(int d, int i, int j, int k) const {
    return cent ? cent[c(i, j, k) + d * int64_t(n[0]) * n[1] * n[2]] : 0.0;
  }
  __device__ __forceinline__ double a(int d, int i, int j, int k) const { return ap[d][f(d, i, j, k)]; }
  __device__ __forceinline__ double fcv(int d, int comp, int i, int j, int k) const {
    return fc[d][f(d, i, j, k) + comp * fn(d)];
  }
};

struct EBWork {
  Space s;  // bx grown by 5 (MOL) or 6 (Godunov), +1 face layer
  double *q, *sl[3], *ft[3], *qf[3], *divu, *divc, *wt, *optmp, *delm, *wtinv;
  // Godunov (CTU-PLM) only: edge states, first-pass and D|E flux records
  double *sm[3], *sp[3], *f1[3], *f2[6];
  // state redistribution only: packed neighbourhood (count in bits 0-3,
  // offsets of 5 bits each from bit 4), overlap count N, neighbourhood
  // volume, centroid (3), averaged state (NVAR) and limited gradient (3 NVAR)
  unsigned long long* nb;
  double *nov, *vhat, *xhat, *qhat, *grad;
};

__global__ void __launch_bounds__(kEB) k_eb_ctoprim(Region r, EBWork W, EBG G, DFab u, KParams P,
                                                     DevError* err) {
  int i, j, k;
  if (!region_cell(r, etid(), i, j, k)) return;
  const Space& s = W.s;
  if (f_covered(G.fl(i, j, k))) {
    const int64_t at = s.idx(i, j, k);
    for (int n = 0; n < SQ_N; ++n) W.q[at + n * s.sn] = 0.;
    return;
  }
  ctoprim_body(i, j, k, s, u, u, false, P, W.q, nullptr, err);
}

template <int d>
__device__ __forceinline__ void eb_slope_cell(int i, int j, int k, const EBWork& W, const EBG& G,
                                              const KParams& P) {
  const unsigned w = G.fl(i, j, k);
  if (f_covered(w)) return;
  constexpr int e0 = (d == 0), e1 = (d == 1), e2 = (d == 2);
  const bool left_ok = f_conn(w, -e0, -e1, -e2) && !f_covered(G.fl(i - e0, j - e1, k - e2));
  const bool rght_ok = f_conn(w, e0, e1, e2) && !f_covered(G.fl(i + e0, j + e1, k + e2));
  if (left_ok && rght_ok) {
    mol_slope_body<d>(i, j, k, W.s, P, W.q, W.sl[d]);
  } else {
    const int64_t at = W.s.idx(i, j, k);
    for (int n = 0; n < SL_N; ++n) W.sl[d][at + n * W.s.sn] = 0.;
  }
}

__global__ void __launch_bounds__(kEB) k_eb_slope(Region r, EBWork W, EBG G, KParams P) {
  int i, j, k;
  if (!region_cell(r, etid(), i, j, k)) return;
  switch (blockIdx.y) {
    case 0: eb_slope_cell<0>(i, j, k, W, G, P); break;
    case 1: eb_slope_cell<1>(i, j, k, W, G, P); break;
    default: eb_slope_cell<2>(i, j, k, W, G, P); break;
  }
}

template <int d>
__device__ __forceinline__ void eb_face(int i, int j, int k, const EBWork& W, const EBG& G,
                                        const KGeom& g, const KParams& P) {
  constexpr int e0 = (d == 0), e1 = (d == 1), e2 = (d == 2);
  const Space& s = W.s;
  const int64_t at = s.idx(i, j, k);
  if (f_conn(G.fl(i, j, k), -e0, -e1, -e2) && !f_covered(G.fl(i - e0, j - e1, k - e2))) {
    double f[NVAR], qpres, qun;
    mol_edges_cmpflx<d>(i, j, k, s, g, P, W.q, W.sl[d], f, qpres, qun);
    for (int n = 0; n < NVAR; ++n) W.ft[d][at + n * s.sn] = f[n];
    W.qf[d][at] = qpres;
    W.qf[d][at + s.sn] = qun;
  } else {
    // a closed face carries no Riemann flux (artificial viscosity is added
    // to it later); zeroing it here keeps a reused workspace free of the
    // previous evaluation's values
    for (int n = 0; n < NVAR; ++n) W.ft[d][at + n * s.sn] = 0.;
    W.qf[d][at] = 0.;
    W.qf[d][at + s.sn] = 0.;
  }
  W.ft[d][at + UTEMP * s.sn] = 0.0;
}

template <int d>
__device__ __forceinline__ void eb_adjust(int i, int j, int k, const EBWork& W, const EBG& G,
                                          const KGeom& g, const KParams& P, const DFab& u);

__device__ __forceinline__ bool in_region(const Region& r, int i, int j, int k) {
  return i >= r.lo[0] && i < r.lo[0] + r.n[0] && j >= r.lo[1] && j < r.lo[1] + r.n[1] &&
         k >= r.lo[2] && k < r.lo[2] + r.n[2];
}

// Faces of the flux box ra[d] (faces of grow(bx,3)): the Riemann flux on
// the faces of rf[d] (faces of grow(bx,2), transverse +1), zero on the
// outer layer; then adjust_fluxes_eb on every face of ra[d] (its
// artificial viscosity is added to the face's own value, so doing it here
// rather than in a separate pass changes no bits; nodal div u is computed
// before this kernel).
template <int d>
__device__ __forceinline__ void eb_face_or_zero(const Region& rf, int i, int j, int k,
                                                const EBWork& W, const EBG& G, const KGeom& g,
                                                const KParams& P, const DFab& u) {
  if (in_region(rf, i, j, k)) {
    eb_face<d>(i, j, k, W, G, g, P);
  } else {
    const int64_t at = W.s.idx(i, j, k);
    for (int n = 0; n < NVAR; ++n) W.ft[d][at + n * W.s.sn] = 0.;
    W.qf[d][at] = 0.;
    W.qf[d][at + W.s.sn] = 0.;
  }
  eb_adjust<d>(i, j, k, W, G, g, P, u);
}

__global__ void __launch_bounds__(kEB) k_eb_face(Region r0, Region r1, Region r2, Region a0,
                                                  Region a1, Region a2, EBWork W, EBG G,
                                                  KGeom g, KParams P, DFab u) {
  int i, j, k;
  const int64_t t = etid();
  switch (blockIdx.y) {
    case 0: if (region_cell(a0, t, i, j, k)) eb_face_or_zero<0>(r0, i, j, k, W, G, g, P, u); break;
    case 1: if (region_cell(a1, t, i, j, k)) eb_face_or_zero<1>(r1, i, j, k, W, G, g, P, u); break;
    default:
      if (region_cell(a2, t, i, j, k)) eb_face_or_zero<2>(r2, i, j, k, W, G, g, P, u);
      break;
  }
}

// eb_divu (Hydro_utils_eb_K.H:31-78) at node (i,j,k).
__global__ void __launch_bounds__(kEB) k_eb_divu(Region r, EBWork W, EBG G, KGeom g) {
  int i, j, k;
  if (!region_cell(r, etid(), i, j, k)) return;
  const Space& s = W.s;
  const double surrounding_vol = G.vf(i, j, k) + G.vf(i - 1, j, k) + G.vf(i, j - 1, k) +
                                 G.vf(i - 1, j - 1, k) + G.vf(i, j, k - 1) +
                                 G.vf(i - 1, j, k - 1) + G.vf(i, j - 1, k - 1) +
                                 G.vf(i - 1, j - 1, k - 1);
  const double cutoff = 8.0 * (1.0 - 1.e-12);
  double dv = 0.0;
  if (surrounding_vol >= cutoff) {
    auto Q = [&](int ii, int jj, int kk, int n) { return W.q[s.idx(ii, jj, kk) + n * s.sn]; };
    const double dxinv0 = 1. / g.dx[0], dxinv1 = 1. / g.dx[1], dxinv2 = 1. / g.dx[2];
    const double ux = 0.25 *
        (Q(i, j, k, SQ_U) - Q(i - 1, j, k, SQ_U) + Q(i, j, k - 1, SQ_U) -
         Q(i - 1, j, k - 1, SQ_U) + Q(i, j - 1, k, SQ_U) - Q(i - 1, j - 1, k, SQ_U) +
         Q(i, j - 1, k - 1, SQ_U) - Q(i - 1, j - 1, k - 1, SQ_U)) * dxinv0;
    const double vy = 0.25 *
        (Q(i, j, k, SQ_V) - Q(i, j - 1, k, SQ_V) + Q(i, j, k - 1, SQ_V) -
         Q(i, j - 1, k - 1, SQ_V) + Q(i - 1, j, k, SQ_V) - Q(i - 1, j - 1, k, SQ_V) +
         Q(i - 1, j, k - 1, SQ_V) - Q(i - 1, j - 1, k - 1, SQ_V)) * dxinv1;
    const double wz = 0.25 *
        (Q(i, j, k, SQ_W) - Q(i, j, k - 1, SQ_W) + Q(i - 1, j, k, SQ_W) -
         Q(i - 1, j, k - 1, SQ_W) + Q(i, j - 1, k, SQ_W) - Q(i, j - 1, k - 1, SQ_W) +
         Q(i - 1, j - 1, k, SQ_W) - Q(i - 1, j - 1, k - 1, SQ_W)) * dxinv2;
    dv = ux + vy + wz;
  }
  W.divu[s.idx(i, j, k)] = dv;
}

// adjust_fluxes_eb on one face: hydro_artif_visc, then (open faces)
// hydro_norm_spec_flx and hydro_ext_flx_eb.
template <int d>
__device__ __forceinline__ void eb_adjust(int i, int j, int k, const EBWork& W, const EBG& G,
                                          const KGeom& g, const KParams& P, const DFab& u) {
  const Space& s = W.s;
  constexpr int e0 = (d == 0), e1 = (d == 1), e2 = (d == 2);
  constexpr int t1 = (d == 0) ? 1 : 0;
  constexpr int t2 = (d == 2) ? 1 : 2;
  const int64_t st1 = (t1 == 0) ? 1 : (t1 == 1) ? s.sy : s.sz;
  const int64_t st2 = (t2 == 0) ? 1 : (t2 == 1) ? s.sy : s.sz;
  const int64_t at = s.idx(i, j, k);
  double* fx = W.ft[d];
  const double div = P.difmag * dmin(0.0, 0.25 * (W.divu[at] + W.divu[at + st1] +
                                                   W.divu[at + st2] + W.divu[at + st1 + st2]));
  const int idx = (d == 0) ? i : (d == 1) ? j : k;
  const bool at_bndry = (idx == g.dlo[d] && g.bclo[d] == CAMR_BC_NOSLIPWALL) ||
                        (idx == g.dhi[d] + 1 && g.bchi[d] == CAMR_BC_NOSLIPWALL);
  for (int n = 0; n < NVAR; ++n) {
    if (n == UTEMP) continue;
    const bool is_tang_vel = (d == 0 && (n == UMY || n == UMZ)) ||
                             (d == 1 && (n == UMX || n == UMZ)) ||
                             (d == 2 && (n == UMX || n == UMY));
    if (!(at_bndry && is_tang_vel))
      fx[at + n * s.sn] += g.dx[d] * div * (u(i, j, k, n) - u(i - e0, j - e1, k - e2, n));
  }
  fx[at + UTEMP * s.sn] = 0.0;
  if (G.a(d, i, j, k) > 0.) {
    double summ = 0.0;
    for (int n = UFS; n < UFS + NSPEC; ++n) summ += fx[at + n * s.sn];
    const double fac = (summ != 0.0) ? fx[at + URHO * s.sn] / summ : 1.0;
    for (int n = UFS; n < UFS + NSPEC; ++n) fx[at + n * s.sn] *= fac;
    const double areafac = (d == 0) ? g.dx[1] * g.dx[2] : (d == 1) ? g.dx[0] * g.dx[2]
                                                                   : g.dx[1] * g.dx[0];
    for (int n = 0; n < NVAR; ++n) fx[at + n * s.sn] *= areafac;
  }
}

// Value of face array `a` (component comp of stride sn) at the centroid of
// face (i,j,k) of direction d: bilinear blend with the neighbouring faces in
// the transverse directions the centroid leans to, when connected.
template <int d>
__device__ __forceinline__ double face_centroid_value(const double* a, const Space& s,
                                                      const EBG& G, int i, int j, int k,
                                                      double aval) {
  const double apv = G.a(d, i, j, k);
  if (apv != 0.0 && apv != 1.0) {
    constexpr int ta = (d == 0) ? 1 : 0;  // first transverse direction
    constexpr int tb = (d == 2) ? 1 : 2;  // second
    const double c0 = G.fcv(d, 0, i, j, k), c1 = G.fcv(d, 1, i, j, k);
    const int oa = static_cast<int>(copysign(1.0, c0));
    const int ob = static_cast<int>(copysign(1.0, c1));
    int da[3] = {0, 0, 0}, db[3] = {0, 0, 0};
    da[ta] = oa;
    db[tb] = ob;
    const unsigned w = G.fl(i, j, k);
    const double fa = f_conn(w, da[0], da[1], da[2]) ? fabs(c0) : 0.0;
    const double fb = f_conn(w, db[0], db[1], db[2]) ? fabs(c1) : 0.0;
    const double va = a[s.idx(i + da[0], j + da[1], k + da[2])];
    const double vb = a[s.idx(i + db[0], j + db[1], k + db[2])];
    const double vab = a[s.idx(i + da[0] + db[0], j + da[1] + db[1], k + da[2] + db[2])];
    aval = (1.0 - fa) * (1.0 - fb) * aval + fa * (1.0 - fb) * va + fb * (1.0 - fa) * vb +
           fa * fb * vab;
  }
  return aval;
}

// Normal velocity at the centroid of face (ii,jj,kk) of direction dd from
// the interface records (p, u_n) of the faces, or 0 on a closed face
// (eb_pdivu, Hydro_utils_eb_K.H:171-270).
template <int dd>
__device__ __forceinline__ double pdivu_face(const double* qq, const Space& s, const EBG& G,
                                             int ii, int jj, int kk) {
  if (G.a(dd, ii, jj, kk) > 0.0)
    return face_centroid_value<dd>(qq + s.sn, s, G, ii, jj, kk, qq[s.idx(ii, jj, kk) + s.sn]);
  return 0.0;
}

// compute_hyp_wallflux (Hydro_hypflux_eb_K.H): the flux through the EB wall
// of a cut cell from the Riemann problem (u_n, -u_n) with the wall normal
// given by the area-fraction differences.
__device__ __forceinline__ void wall_flux(const double* q, const Space& s, int64_t at,
                                          double axm, double axp, double aym, double ayp,
                                          double azm, double azp, const KParams& P,
                                          double* fw) {
  const double u = q[at + SQ_U * s.sn];
  const double v = q[at + SQ_V * s.sn];
  const double w = q[at + SQ_W * s.sn];
  const double apnorm = sqrt((axm - axp) * (axm - axp) + (aym - ayp) * (aym - ayp) +
                             (azm - azp) * (azm - azp));
  const double apnorminv = 1. / apnorm;
  const double un = u * (axm - axp) * apnorminv + v * (aym - ayp) * apnorminv +
                    w * (azm - azp) * apnorminv;
  const double rho = q[at + SQ_RHO * s.sn];
  const double p = q[at + SQ_P * s.sn];
  const double qrei = q[at + SQ_REINT * s.sn];
  const double gamc = P.gamma;
  const double cav = q[at + SQ_C * s.sn];
  const double smallc = q[at + SQ_CSML * s.sn];
  const ROut o = riemannus(rho, un, 0., 0., p, qrei, rho, -un, 0., 0., p, qrei, cav, gamc, gamc,
                           P.small, smallc, P.small_dens, P.small_pres, P.smallu);
  for (int n = 0; n < NVAR; ++n) fw[n] = 0.;
  fw[URHO] = o.f_rho;
  fw[UEDEN] = o.f_eden;
  fw[UEINT] = o.f_eint;
  fw[UMX] = (axm - axp) * o.f_un;
  fw[UMY] = (aym - ayp) * o.f_un;
  fw[UMZ] = (azm - azp) * o.f_un;
}

// eb_compute_div for all components + eb_pdivu + the redistribution weight
// of one cell of grow(bx,2); writes the face-centroid fluxes of bx's faces.
__global__ void __launch_bounds__(kEB) k_eb_div(Region r, EBWork W, EBG G, KGeom g, KParams P,
                                                 DFab fo0, DFab fo1, DFab fo2, int wtype) {
  int i, j, k;
  if (!region_cell(r, etid(), i, j, k)) return;
  const unsigned w = G.fl(i, j, k);
  if (f_covered(w)) return;
  const Space& s = W.s;
  const int64_t at = s.idx(i, j, k);
  const bool valid_cell = fo0.p && g.lo[0] <= i && i <= g.hi[0] && g.lo[1] <= j &&
                          j <= g.hi[1] && g.lo[2] <= k && k <= g.hi[2];
  const bool x_high = (i == g.hi[0]), y_high = (j == g.hi[1]), z_high = (k == g.hi[2]);
  const double dxinv0 = 1. / g.dx[0], dxinv1 = 1. / g.dx[1], dxinv2 = 1. / g.dx[2];
  const double cell_vol_inv = dxinv0 * dxinv1 * dxinv2;
  const double* fx = W.ft[0];
  const double* fy = W.ft[1];
  const double* fz = W.ft[2];
  const int64_t sx = 1, sy = s.sy, sz = s.sz;
  if (f_regular(w)) {
    for (int n = 0; n < NVAR; ++n) {
      const int64_t o = at + n * s.sn;
      double dv = cell_vol_inv * (fx[o + sx] - fx[o]) + cell_vol_inv * (fy[o + sy] - fy[o]) +
                  cell_vol_inv * (fz[o + sz] - fz[o]);
      W.divc[o] = dv * -1.0;
      if (valid_cell) {
        fo0(i, j, k, n) = fx[o];
        fo1(i, j, k, n) = fy[o];
        fo2(i, j, k, n) = fz[o];
        if (x_high) fo0(i + 1, j, k, n) = fx[o + sx];
        if (y_high) fo1(i, j + 1, k, n) = fy[o + sy];
        if (z_high) fo2(i, j, k + 1, n) = fz[o + sz];
      }
    }
  } else {
    double fw[NVAR];
    wall_flux(W.q, s, at, G.a(0, i, j, k), G.a(0, i + 1, j, k), G.a(1, i, j, k),
              G.a(1, i, j + 1, k), G.a(2, i, j, k), G.a(2, i, j, k + 1), P, fw);
    const double vfc = G.vf(i, j, k);
    for (int n = 0; n < NVAR; ++n) {
      const int64_t o = at + n * s.sn;
      const double* ax = fx + n * s.sn;
      const double* ay = fy + n * s.sn;
      const double* az = fz + n * s.sn;
      const double fxm = face_centroid_value<0>(ax, s, G, i, j, k, fx[o]);
      const double fxp = face_centroid_value<0>(ax, s, G, i + 1, j, k, fx[o + sx]);
      const double fym = face_centroid_value<1>(ay, s, G, i, j, k, fy[o]);
      const double fyp = face_centroid_value<1>(ay, s, G, i, j + 1, k, fy[o + sy]);
      const double fzm = face_centroid_value<2>(az, s, G, i, j, k, fz[o]);
      const double fzp = face_centroid_value<2>(az, s, G, i, j, k + 1, fz[o + sz]);
      if (valid_cell) {
        fo0(i, j, k, n) = fxm;
        fo1(i, j, k, n) = fym;
        fo2(i, j, k, n) = fzm;
        if (x_high) fo0(i + 1, j, k, n) = fxp;
        if (y_high) fo1(i, j + 1, k, n) = fyp;
        if (z_high) fo2(i, j, k + 1, n) = fzp;
      }
      double dv = cell_vol_inv / vfc *
                  (G.a(0, i + 1, j, k) * fxp - G.a(0, i, j, k) * fxm + G.a(1, i, j + 1, k) * fyp -
                   G.a(1, i, j, k) * fym + G.a(2, i, j, k + 1) * fzp - G.a(2, i, j, k) * fzm);
      dv += fw[n] * dxinv0 / vfc;
      W.divc[o] = dv * -1.0;
    }
  }
  // p div u (eb_pdivu)
  const double* q1 = W.qf[0];
  const double* q2 = W.qf[1];
  const double* q3 = W.qf[2];
  const int64_t sn = s.sn;
  if (f_regular(w)) {
    const double pdivu =
        0.5 * ((q1[at + sx] + q1[at]) * (q1[at + sx + sn] - q1[at + sn]) * dxinv0 +
               (q2[at + sy] + q2[at]) * (q2[at + sy + sn] - q2[at + sn]) * dxinv1 +
               (q3[at + sz] + q3[at]) * (q3[at + sz + sn] - q3[at + sn]) * dxinv2);
    W.divc[at + UEINT * sn] -= pdivu;
  } else {
    const double fxm = pdivu_face<0>(q1, s, G, i, j, k), fxp = pdivu_face<0>(q1, s, G, i + 1, j, k);
    const double fym = pdivu_face<1>(q2, s, G, i, j, k), fyp = pdivu_face<1>(q2, s, G, i, j + 1, k);
    const double fzm = pdivu_face<2>(q3, s, G, i, j, k), fzp = pdivu_face<2>(q3, s, G, i, j, k + 1);
    W.divc[at + UEINT * sn] -=
        (1.0 / G.vf(i, j, k)) * W.q[at + SQ_P * sn] *
        (dxinv0 * (G.a(0, i + 1, j, k) * fxp - G.a(0, i, j, k) * fxm) +
         dxinv1 * (G.a(1, i, j + 1, k) * fyp - G.a(1, i, j, k) * fym) +
         dxinv2 * (G.a(2, i, j, k + 1) * fzp - G.a(2, i, j, k) * fzm));
  }
  double wv;
  if (wtype == 0) {
    wv = 1.0;
  } else if (wtype == 1) {
    const double uu = W.q[at + SQ_U * sn], vv = W.q[at + SQ_V * sn], ww = W.q[at + SQ_W * sn];
    wv = W.q[at + SQ_RHO * sn] * (W.q[at + SQ_REINT * sn] + 0.5 * (uu * uu + vv * vv + ww * ww));
  } else if (wtype == 2) {
    wv = W.q[at + SQ_RHO * sn];
  } else {
    wv = G.vf(i, j, k);
  }
  W.wt[at] = wv;
}

// Domain grown by 2 in its periodic directions (the redistribution's dbox).
struct DBox {
  int lo[3], hi[3];
  __device__ __forceinline__ bool has(int i, int j, int k) const {
    return i >= lo[0] && i <= hi[0] && j >= lo[1] && j <= hi[1] && k >= lo[2] && k <= hi[2];
  }
};

// Flux redistribution, part 1 (cut cells of grow(bx,1)): divnc, the
// cell's own correction optmp and the mass delm it sends, and the inverse
// of its neighbourhood weight.
__global__ void __launch_bounds__(kEB) k_eb_redist1(Region r, EBWork W, EBG G, DBox db) {
  int i, j, k;
  if (!region_cell(r, etid(), i, j, k)) return;
  const unsigned w = G.fl(i, j, k);
  const Space& s = W.s;
  const int64_t at = s.idx(i, j, k);
  if (!f_single(w)) {
    for (int n = 0; n < NVAR; ++n) W.delm[at + n * s.sn] = 0.0;
    return;
  }
  double wtot = 0.0;
  for (int kk = -1; kk <= 1; ++kk)
    for (int jj = -1; jj <= 1; ++jj)
      for (int ii = -1; ii <= 1; ++ii)
        if (f_conn(w, ii, jj, kk) && db.has(i + ii, j + jj, k + kk))
          wtot += G.vf(i + ii, j + jj, k + kk) * W.wt[s.idx(i + ii, j + jj, k + kk)];
  W.wtinv[at] = 1.0 / wtot;
  for (int n = 0; n < NVAR; ++n) {
    double divnc = 0.0, vtot = 0.0;
    for (int kk = -1; kk <= 1; ++kk)
      for (int jj = -1; jj <= 1; ++jj)
        for (int ii = -1; ii <= 1; ++ii)
          if (f_conn(w, ii, jj, kk) && db.has(i + ii, j + jj, k + kk)) {
            const double wf = G.vf(i + ii, j + jj, k + kk);
            vtot += wf;
            divnc += wf * W.divc[s.idx(i + ii, j + jj, k + kk) + n * s.sn];
          }
    divnc /= vtot;
    const double vfc = G.vf(i, j, k);
    const double op = (1.0 - vfc) * (divnc - W.divc[at + n * s.sn]);
    W.optmp[at + n * s.sn] = op;
    W.delm[at + n * s.sn] = -vfc * op;
  }
}

// Part 2 (cells of bx): gather the mass the cut cells of the neighbourhood
// send (senders in raster order), and the final dSdt.
__global__ void __launch_bounds__(kEB) k_eb_redist2(Region r, EBWork W, EBG G, DBox db,
                                                     KGeom g, DFab dsdt, int redist) {
  int i, j, k;
  if (!region_cell(r, etid(), i, j, k)) return;
  const Space& s = W.s;
  const int64_t at = s.idx(i, j, k);
  const unsigned wc = G.fl(i, j, k);
  if (f_covered(wc)) {
    for (int n = 0; n < NVAR; ++n) dsdt(i, j, k, n) = 0.0;
    return;
  }
  if (!redist) {
    for (int n = 0; n < NVAR; ++n) dsdt(i, j, k, n) = W.divc[at + n * s.sn];
    return;
  }
  // the cut cells that send to this cell, in raster order (most cells
  // have none: they take divc, plus their own correction if cut)
  int64_t from[27];
  int nfrom = 0;
  if (db.has(i, j, k)) {
    for (int kk = -1; kk <= 1; ++kk)
      for (int jj = -1; jj <= 1; ++jj)
        for (int ii = -1; ii <= 1; ++ii) {
          const int si = i + ii, sj = j + jj, sk = k + kk;
          if (si < g.lo[0] - 1 || si > g.hi[0] + 1 || sj < g.lo[1] - 1 || sj > g.hi[1] + 1 ||
              sk < g.lo[2] - 1 || sk > g.hi[2] + 1)
            continue;
          const unsigned ws = G.fl(si, sj, sk);
          if (!f_single(ws) || !f_conn(ws, -ii, -jj, -kk)) continue;
          from[nfrom++] = s.idx(si, sj, sk);
        }
  }
  const bool own = f_single(wc);
  if (!own && nfrom == 0) {
    for (int n = 0; n < NVAR; ++n) dsdt(i, j, k, n) = W.divc[at + n * s.sn] + 0.0;
    return;
  }
  const double wtc = W.wt[at];
  for (int n = 0; n < NVAR; ++n) {
    double acc = own ? W.optmp[at + n * s.sn] : 0.0;
    for (int q = 0; q < nfrom; ++q) {
      const int64_t as = from[q];
      acc += W.delm[as + n * s.sn] * W.wtinv[as] * wtc;
    }
    dsdt(i, j, k, n) = W.divc[at + n * s.sn] + acc;
  }
}

__global__ void __launch_bounds__(kEB) k_eb_zero_faces(Region r, DFab f) {
  int i, j, k;
  if (!region_cell(r, etid(), i, j, k)) return;
  for (int n = 0; n < NVAR; ++n) f(i, j, k, n) = 0.0;
}


// ---------------------------------------------------------------------------
// Godunov (CTU-PLM) with embedded boundaries: Godunov_umeth_eb
// (Godunov/Godunov_3D_eb.cpp:16-565) as face-centred passes.  The reference
// runs transdo/transdd per cell and fills both faces of the cell; here a
// face thread evaluates the half it needs of each of its two cells (on an
// open face both of them are uncovered, so the reference's lo/hi-face
// guards hold and only its no_cov_face guard, which zeroes the transverse
// terms, remains).

// flatten_eb (Godunov/flatten.H:104-134) of cell (i,j,k) in direction d:
// 1 when the +-3 stencil leaves the q box or meets a cut cell
// (is_cut_neighborhood, EB/eb_utils.H:7-20), else flatten.
template <int d>
__device__ __forceinline__ double flatten_eb_dir(int i, int j, int k, const EBWork& W,
                                                 const EBG& G, const Region& qbox) {
  constexpr int e0 = (d == 0), e1 = (d == 1), e2 = (d == 2);
  if (!in_region(qbox, i + 3 * e0, j + 3 * e1, k + 3 * e2) ||
      !in_region(qbox, i - 3 * e0, j - 3 * e1, k - 3 * e2))
    return 1.0;
  bool cut = f_single(G.fl(i, j, k));
  for (int n = 1; n <= 3; ++n)
    cut = cut || f_single(G.fl(i - n * e0, j - n * e1, k - n * e2)) ||
          f_single(G.fl(i + n * e0, j + n * e1, k + n * e2));
  if (cut) return 1.0;
  const Space& s = W.s;
  const int64_t at = s.idx(i, j, k);
  const int64_t st = (d == 0) ? 1 : (d == 1) ? s.sy : s.sz;
  double pp[7], un[7];
  for (int o = -3; o <= 3; ++o) {
    pp[o + 3] = W.q[at + o * st + SQ_P * s.sn];
    un[o + 3] = W.q[at + o * st + (SQ_U + d) * s.sn];
  }
  return flatten_dir(pp, un);
}

// PLM predictor of one uncovered cell in direction d (Godunov_3D_eb.cpp:
// 95-149): flattening, plm_slope_eb (PLM_eb.H:18-58: 4th order when the
// cells at +-1, +-2 are uncovered, 2nd order at +-1, else 0), then
// hydro_plm_d_eb (PLM_eb.H:111-286: a face with zero area gets a zero state).
template <int d>
__device__ __forceinline__ void ebc_trace_cell(int i, int j, int k, const EBWork& W,
                                               const EBG& G, const KGeom& g, const KParams& P,
                                               double dt, const Region& qbox) {
  if (f_covered(G.fl(i, j, k))) return;
  constexpr int e0 = (d == 0), e1 = (d == 1), e2 = (d == 2);
  const Space& s = W.s;
  const int64_t at = s.idx(i, j, k);
  const int64_t st = (d == 0) ? 1 : (d == 1) ? s.sy : s.sz;
  double fl = 1.0;
  if (P.use_flattening == 1) {
    fl = dmin(fl, flatten_eb_dir<0>(i, j, k, W, G, qbox));
    fl = dmin(fl, flatten_eb_dir<1>(i, j, k, W, G, qbox));
    fl = dmin(fl, flatten_eb_dir<2>(i, j, k, W, G, qbox));
  }
  auto open = [&](int o) { return !f_covered(G.fl(i + o * e0, j + o * e1, k + o * e2)); };
  int order = 0;
  if (P.plm_iorder == 4 && open(-1) && open(-2) && open(1) && open(2)) {
    order = 4;
  } else if (P.plm_iorder > 1 && open(-1) && open(1)) {
    order = 2;
  }
  double slope[ES_N];
  const int slot_of[ES_N] = {SQ_RHO, SQ_U, SQ_V, SQ_W, SQ_P, SQ_REINT, SQ_FS, SQ_FS + 1,
                             SQ_FS + 2};
  for (int n = 0; n < ES_N; ++n) {
    if (order == 0) {
      slope[n] = 0.0;
      continue;
    }
    const double* qq = W.q + slot_of[n] * s.sn;
    slope[n] = plm_slope(qq[at - 2 * st], qq[at - st], qq[at], qq[at + st], qq[at + 2 * st], fl,
                         order);
  }
  if (P.use_pslope && order > 0) {
    // plm_pslope_eb (PLM_eb.H:63-104) with the zero predictor sources of an
    // EB Godunov step
    double pv[5], rv[5], su[5];
    for (int o = 0; o < 5; ++o) {
      pv[o] = W.q[at + (o - 2) * st + SQ_P * s.sn];
      rv[o] = W.q[at + (o - 2) * st + SQ_RHO * s.sn];
      su[o] = 0.0;
    }
    slope[ES_P] = plm_pslope(pv, rv, su, g.dx[d], fl, order);
  }
  double qp_o[ES_N], qm_o[ES_N];
  plm_edge_states<d>(W.q, at, s.sn, slope, dt / g.dx[d], P, qp_o, qm_o);
  if (!(G.a(d, i, j, k) > 0.0))
    for (int n = 0; n < ES_N; ++n) qp_o[n] = 0.0;
  if (!(G.a(d, i + e0, j + e1, k + e2) > 0.0))
    for (int n = 0; n < ES_N; ++n) qm_o[n] = 0.0;
  store_es(W.sp[d], s, at, qp_o);
  store_es(W.sm[d], s, at + st, qm_o);
}

__global__ void __launch_bounds__(kEB) k_ebc_trace(Region r, EBWork W, EBG G, KGeom g, KParams P,
                                                    DtRef dtr, Region qbox) {
  int i, j, k;
  if (!region_cell(r, etid(), i, j, k)) return;
  const double dt = dtr.get();
  switch (blockIdx.y) {
    case 0: ebc_trace_cell<0>(i, j, k, W, G, g, P, dt, qbox); break;
    case 1: ebc_trace_cell<1>(i, j, k, W, G, g, P, dt, qbox); break;
    default: ebc_trace_cell<2>(i, j, k, W, G, g, P, dt, qbox); break;
  }
}

__device__ __forceinline__ void store_fr(double* o, const Space& s, int64_t at, const double* f,
                                         double qpres, double qun) {
  o[at + FR_RHO * s.sn] = f[URHO];
  o[at + FR_MX * s.sn] = f[UMX];
  o[at + FR_MY * s.sn] = f[UMY];
  o[at + FR_MZ * s.sn] = f[UMZ];
  o[at + FR_E * s.sn] = f[UEDEN];
  for (int sp = 0; sp < NSPEC; ++sp) o[at + (FR_FS + sp) * s.sn] = f[UFS + sp];
  o[at + FR_PRES * s.sn] = qpres;
  o[at + FR_UN * s.sn] = qun;
}

__device__ __forceinline__ void zero_fr(double* o, const Space& s, int64_t at) {
  for (int n = 0; n < FR_N; ++n) o[at + n * s.sn] = 0.0;
}

// First-pass Riemann flux on an open E-face (Godunov_3D_eb.cpp:157-210).
template <int E>
__device__ __forceinline__ void ebc_flux1_face(int i, int j, int k, const EBWork& W,
                                               const EBG& G, const KGeom& g, const KParams& P) {
  const Space& s = W.s;
  const int64_t at = s.idx(i, j, k);
  if (!(G.a(E, i, j, k) > 0.0)) {
    zero_fr(W.f1[E], s, at);
    return;
  }
  const int64_t stE = (E == 0) ? 1 : (E == 1) ? s.sy : s.sz;
  double qm[ES_N], qp[ES_N];
  load_es(W.sm[E], s, at, qm);
  load_es(W.sp[E], s, at, qp);
  const CellAux aL = load_aux(W.q, s, at - stE, P.gamma);
  const CellAux aR = load_aux(W.q, s, at, P.gamma);
  const int idx = (E == 0) ? i : (E == 1) ? j : k;
  double f[NVAR], qpres, qun;
  cmpflx<E>(qm, qp, aL, aR, idx, g.bclo[E], g.bchi[E], g.dlo[E], g.dhi[E], P, f, qpres, qun);
  store_fr(W.f1[E], s, at, f, qpres, qun);
}

__global__ void __launch_bounds__(kEB) k_ebc_flux1(Region r0, Region r1, Region r2, EBWork W,
                                                    EBG G, KGeom g, KParams P) {
  int i, j, k;
  const int64_t t = etid();
  switch (blockIdx.y) {
    case 0: if (region_cell(r0, t, i, j, k)) ebc_flux1_face<0>(i, j, k, W, G, g, P); break;
    case 1: if (region_cell(r1, t, i, j, k)) ebc_flux1_face<1>(i, j, k, W, G, g, P); break;
    default: if (region_cell(r2, t, i, j, k)) ebc_flux1_face<2>(i, j, k, W, G, g, P); break;
  }
}

__device__ __forceinline__ TTerms zero_tterms() {
  TTerms t;
  t.flxrho = t.flxu = t.flxv = t.flxw = t.flxe = 0.0;
  for (int n = 0; n < NSPEC; ++n) t.compn[n] = 0.0;
  t.dAup = t.pav = t.dAu = 0.0;
  return t;
}

__device__ __forceinline__ TDTerms zero_tdterms() {
  TDTerms t;
  t.flxrho = t.flxu = t.flxv = t.flxw = t.flxe = 0.0;
  for (int n = 0; n < NSPEC; ++n) t.compn[n] = 0.0;
  t.pxnew = t.pynew = 0.0;
  return t;
}

// D|E pass on an open D-face: the D-states of both adjacent cells corrected
// by their E-flux differences (hydro_transdo, Godunov_utils_3D.H:22-239;
// no_cov_face: both E-faces of the cell open), then the Riemann flux
// (Godunov_3D_eb.cpp:212-409).
template <int D, int E>
__device__ __forceinline__ void ebc_flux2_face(int i, int j, int k, const EBWork& W,
                                               const EBG& G, const KGeom& g, const KParams& P,
                                               double dt) {
  const Space& s = W.s;
  const int64_t at = s.idx(i, j, k);
  double* o = W.f2[combo(D, E)];
  if (!(G.a(D, i, j, k) > 0.0)) {
    zero_fr(o, s, at);
    return;
  }
  constexpr int d0 = (D == 0), d1 = (D == 1), d2 = (D == 2);
  constexpr int e0 = (E == 0), e1 = (E == 1), e2 = (E == 2);
  const int64_t stD = (D == 0) ? 1 : (D == 1) ? s.sy : s.sz;
  const int64_t stE = (E == 0) ? 1 : (E == 1) ? s.sy : s.sz;
  const double cdtdx = 1.0 / 3.0 * dt / g.dx[E];
  const double* fE = W.f1[E];
  double qm[ES_N], qp[ES_N], qn[ES_N];
  {
    const int ci = i - d0, cj = j - d1, ck = k - d2;
    const bool ncf = G.a(E, ci + e0, cj + e1, ck + e2) > 0.0 && G.a(E, ci, cj, ck) > 0.0;
    TTerms t = zero_tterms();
    if (ncf) {
      double lo[FR_N], hi[FR_N];
      load_fr(fE, s, at - stD, lo);
      load_fr(fE, s, at - stD + stE, hi);
      t = transdo_terms(lo, hi, cdtdx);
    }
    load_es(W.sm[D], s, at, qn);
    transdo_side(t, P.gamma, qn, cdtdx, P, qm);
  }
  {
    const bool ncf = G.a(E, i + e0, j + e1, k + e2) > 0.0 && G.a(E, i, j, k) > 0.0;
    TTerms t = zero_tterms();
    if (ncf) {
      double lo[FR_N], hi[FR_N];
      load_fr(fE, s, at, lo);
      load_fr(fE, s, at + stE, hi);
      t = transdo_terms(lo, hi, cdtdx);
    }
    load_es(W.sp[D], s, at, qn);
    transdo_side(t, P.gamma, qn, cdtdx, P, qp);
  }
  const CellAux aL = load_aux(W.q, s, at - stD, P.gamma);
  const CellAux aR = load_aux(W.q, s, at, P.gamma);
  const int idx = (D == 0) ? i : (D == 1) ? j : k;
  double f[NVAR], qpres, qun;
  cmpflx<D>(qm, qp, aL, aR, idx, g.bclo[D], g.bchi[D], g.dlo[D], g.dhi[D], P, f, qpres, qun);
  store_fr(o, s, at, f, qpres, qun);
}

struct Reg6E {
  Region r[6];
};

__global__ void __launch_bounds__(kEB) k_ebc_flux2(Reg6E regs, EBWork W, EBG G, KGeom g,
                                                    KParams P, DtRef dtr) {
  int i, j, k;
  const int64_t t = etid();
  const double dt = dtr.get();
#define CAMR_EBF2(D, E)                                                  \
  case combo(D, E):                                                      \
    if (region_cell(regs.r[combo(D, E)], t, i, j, k))                    \
      ebc_flux2_face<D, E>(i, j, k, W, G, g, P, dt);                     \
    break;
  switch (blockIdx.y) {
    CAMR_EBF2(0, 1)
    CAMR_EBF2(0, 2)
    CAMR_EBF2(1, 0)
    CAMR_EBF2(1, 2)
    CAMR_EBF2(2, 0)
    CAMR_EBF2(2, 1)
    default: break;
  }
#undef CAMR_EBF2
}

// Final pass on an open D-face (Godunov_3D_eb.cpp:421-563): the D-states of
// both cells corrected by the two transverse D|E fluxes (hydro_transdd,
// Godunov_utils_3D.H:245-482, zero sources; no_cov_face: the cell's four
// transverse faces open), then the Riemann flux into the face arrays.
template <int D>
__device__ __forceinline__ void ebc_final_face(int i, int j, int k, const EBWork& W,
                                               const EBG& G, const KGeom& g, const KParams& P,
                                               double dt) {
  const Space& s = W.s;
  const int64_t at = s.idx(i, j, k);
  if (!(G.a(D, i, j, k) > 0.0)) {
    for (int n = 0; n < NVAR; ++n) W.ft[D][at + n * s.sn] = 0.;
    W.qf[D][at] = 0.;
    W.qf[D][at + s.sn] = 0.;
    return;
  }
  constexpr int t0 = (D == 0) ? 1 : 0;
  constexpr int t1 = (D == 2) ? 1 : 2;
  constexpr int d0 = (D == 0), d1 = (D == 1), d2 = (D == 2);
  constexpr int a0 = (t0 == 0), a1 = (t0 == 1), a2 = (t0 == 2);
  constexpr int b0 = (t1 == 0), b1 = (t1 == 1), b2 = (t1 == 2);
  const int64_t stD = (D == 0) ? 1 : (D == 1) ? s.sy : s.sz;
  const int64_t st0 = (t0 == 0) ? 1 : (t0 == 1) ? s.sy : s.sz;
  const int64_t st1 = (t1 == 0) ? 1 : (t1 == 1) ? s.sy : s.sz;
  const double hdt = 0.5 * dt;
  const double cdtdx0 = 0.5 * dt / g.dx[t0];
  const double cdtdx1 = 0.5 * dt / g.dx[t1];
  const double* fa = W.f2[combo(t0, t1)];
  const double* fb = W.f2[combo(t1, t0)];
  double sq[ES_N];
  for (int n = 0; n < ES_N; ++n) sq[n] = 0.0;
  double qm[ES_N], qp[ES_N], qn[ES_N];
  auto ncf_at = [&](int ci, int cj, int ck) {
    return G.a(t0, ci + a0, cj + a1, ck + a2) > 0.0 && G.a(t1, ci + b0, cj + b1, ck + b2) > 0.0 &&
           G.a(t0, ci, cj, ck) > 0.0 && G.a(t1, ci, cj, ck) > 0.0;
  };
  auto terms_at = [&](int64_t cell) {
    double x0[FR_N], x1[FR_N], y0[FR_N], y1[FR_N];
    load_fr(fa, s, cell, x0);
    load_fr(fa, s, cell + st0, x1);
    load_fr(fb, s, cell, y0);
    load_fr(fb, s, cell + st1, y1);
    return transdd_terms(x0, x1, y0, y1, P.gamma, cdtdx0, cdtdx1);
  };
  {
    const TDTerms t = ncf_at(i - d0, j - d1, k - d2) ? terms_at(at - stD) : zero_tdterms();
    load_es(W.sm[D], s, at, qn);
    transdd_side(t, qn, sq, hdt, P, qm);
  }
  {
    const TDTerms t = ncf_at(i, j, k) ? terms_at(at) : zero_tdterms();
    load_es(W.sp[D], s, at, qn);
    transdd_side(t, qn, sq, hdt, P, qp);
  }
  const CellAux aL = load_aux(W.q, s, at - stD, P.gamma);
  const CellAux aR = load_aux(W.q, s, at, P.gamma);
  const int idx = (D == 0) ? i : (D == 1) ? j : k;
  double f[NVAR], qpres, qun;
  cmpflx<D>(qm, qp, aL, aR, idx, g.bclo[D], g.bchi[D], g.dlo[D], g.dhi[D], P, f, qpres, qun);
  for (int n = 0; n < NVAR; ++n) W.ft[D][at + n * s.sn] = f[n];
  W.qf[D][at] = qpres;
  W.qf[D][at + s.sn] = qun;
  W.ft[D][at + UTEMP * s.sn] = 0.0;
}

// Final faces of the flux box ra[d]: the Godunov flux on rf[d], zero on the
// outer layer, then adjust_fluxes_eb (as the MOL face kernel).
template <int d>
__device__ __forceinline__ void ebc_face_or_zero(const Region& rf, int i, int j, int k,
                                                 const EBWork& W, const EBG& G, const KGeom& g,
                                                 const KParams& P, const DFab& u, double dt) {
  if (in_region(rf, i, j, k)) {
    ebc_final_face<d>(i, j, k, W, G, g, P, dt);
  } else {
    const int64_t at = W.s.idx(i, j, k);
    for (int n = 0; n < NVAR; ++n) W.ft[d][at + n * W.s.sn] = 0.;
    W.qf[d][at] = 0.;
    W.qf[d][at + W.s.sn] = 0.;
  }
  eb_adjust<d>(i, j, k, W, G, g, P, u);
}

__global__ void __launch_bounds__(kEB) k_ebc_face(Region r0, Region r1, Region r2, Region a0,
                                                   Region a1, Region a2, EBWork W, EBG G,
                                                   KGeom g, KParams P, DFab u, DtRef dtr) {
  int i, j, k;
  const int64_t t = etid();
  const double dt = dtr.get();
  switch (blockIdx.y) {
    case 0:
      if (region_cell(a0, t, i, j, k)) ebc_face_or_zero<0>(r0, i, j, k, W, G, g, P, u, dt);
      break;
    case 1:
      if (region_cell(a1, t, i, j, k)) ebc_face_or_zero<1>(r1, i, j, k, W, G, g, P, u, dt);
      break;
    default:
      if (region_cell(a2, t, i, j, k)) ebc_face_or_zero<2>(r2, i, j, k, W, G, g, P, u, dt);
      break;
  }
}

// ---------------------------------------------------------------------------
// State redistribution (redist = 2), restated from Berger & Giuliani's
// published method (J. Comput. Phys. 434 (2021) 110205), AMReX's own
// StateRedist being unavailable; the neighbourhood rule is this library's:
// a cut cell with volume fraction under 1/2 merges with connected,
// uncovered neighbours inside the domain, in decreasing order of
// (m . o) / |o| (m = (ap_x(i+1) - ap_x(i), ...) points into the fluid, o is
// the neighbour offset, ties in raster order) until the merged volume
// fraction reaches 1/2 or 8 cells.  Then per neighbourhood the overlap-
// weighted average of U* = U + dt dSdt_pre and its centroid, a limited
// least-squares gradient, and per cell the average over the neighbourhoods
// that hold it.  Conservative; every sum runs in a fixed order, so the
// result is deterministic.
constexpr int kSrdMax = 8;

__device__ __forceinline__ int nb_count(unsigned long long w) { return int(w & 15ull); }
__device__ __forceinline__ int nb_off(unsigned long long w, int c) {
  return int((w >> (4 + 5 * c)) & 31ull);
}
__device__ __forceinline__ bool nb_holds(unsigned long long w, int o) {
  const int n = nb_count(w);
  for (int c = 0; c < n; ++c)
    if (nb_off(w, c) == o) return true;
  return false;
}
__device__ __forceinline__ void off3(int o, int& di, int& dj, int& dk) {
  di = o % 3 - 1;
  dj = (o / 3) % 3 - 1;
  dk = o / 9 - 1;
}

// Neighbourhoods of the cells of grow(bx,4).
__global__ void __launch_bounds__(kEB) k_srd_nbhd(Region r, EBWork W, EBG G, DBox din) {
  int i, j, k;
  if (!region_cell(r, etid(), i, j, k)) return;
  const int64_t at = W.s.idx(i, j, k);
  const unsigned w = G.fl(i, j, k);
  if (f_covered(w) || !din.has(i, j, k)) {
    W.nb[at] = 0ull;
    return;
  }
  unsigned long long out = 1ull | (13ull << 4);
  if (f_single(w) && G.vf(i, j, k) < 0.5) {
    const double m0 = G.a(0, i + 1, j, k) - G.a(0, i, j, k);
    const double m1 = G.a(1, i, j + 1, k) - G.a(1, i, j, k);
    const double m2 = G.a(2, i, j, k + 1) - G.a(2, i, j, k);
    int cand[26];
    double score[26];
    int nc = 0;
    for (int kk = -1; kk <= 1; ++kk)
      for (int jj = -1; jj <= 1; ++jj)
        for (int ii = -1; ii <= 1; ++ii) {
          if (ii == 0 && jj == 0 && kk == 0) continue;
          if (!f_conn(w, ii, jj, kk)) continue;
          if (f_covered(G.fl(i + ii, j + jj, k + kk))) continue;
          if (!din.has(i + ii, j + jj, k + kk)) continue;
          const double len = sqrt(double(ii * ii + jj * jj + kk * kk));
          const double sc = (m0 * ii + m1 * jj + m2 * kk) / len;
          int pos = nc;
          while (pos > 0 && score[pos - 1] < sc) {
            score[pos] = score[pos - 1];
            cand[pos] = cand[pos - 1];
            --pos;
          }
          score[pos] = sc;
          cand[pos] = (ii + 1) + 3 * (jj + 1) + 9 * (kk + 1);
          ++nc;
        }
    double vol = G.vf(i, j, k);
    int n = 1;
    for (int c = 0; c < nc && vol < 0.5 && n < kSrdMax; ++c) {
      int di, dj, dk;
      off3(cand[c], di, dj, dk);
      out |= (unsigned long long)(cand[c]) << (4 + 5 * n);
      ++n;
      vol += G.vf(i + di, j + dj, k + dk);
    }
    out = (out & ~15ull) | (unsigned long long)(n);
  }
  W.nb[at] = out;
}

// Overlap counts N on grow(bx,3).
__global__ void __launch_bounds__(kEB) k_srd_count(Region r, EBWork W, EBG G, DBox din) {
  int i, j, k;
  if (!region_cell(r, etid(), i, j, k)) return;
  const Space& s = W.s;
  const int64_t at = s.idx(i, j, k);
  if (f_covered(G.fl(i, j, k)) || !din.has(i, j, k)) {
    W.nov[at] = 0.0;
    return;
  }
  double cnt = 0.0;
  for (int kk = -1; kk <= 1; ++kk)
    for (int jj = -1; jj <= 1; ++jj)
      for (int ii = -1; ii <= 1; ++ii)
        if (nb_holds(W.nb[s.idx(i - ii, j - jj, k - kk)], (ii + 1) + 3 * (jj + 1) + 9 * (kk + 1)))
          cnt += 1.0;
  W.nov[at] = cnt;
}

// Neighbourhood volume, centroid and averaged state on grow(bx,2).
__global__ void __launch_bounds__(kEB) k_srd_qhat(Region r, EBWork W, EBG G, DFab u, DtRef dtr) {
  int i, j, k;
  if (!region_cell(r, etid(), i, j, k)) return;
  const Space& s = W.s;
  const int64_t at = s.idx(i, j, k);
  const unsigned long long nw = W.nb[at];
  const int nn = nb_count(nw);
  if (nn == 0) return;
  const double dt = dtr.get();
  double v = 0.0, x0 = 0.0, x1 = 0.0, x2 = 0.0;
  double q[NVAR];
  for (int n = 0; n < NVAR; ++n) q[n] = 0.0;
  for (int c = 0; c < nn; ++c) {
    int di, dj, dk;
    off3(nb_off(nw, c), di, dj, dk);
    const int a = i + di, b = j + dj, cc = k + dk;
    const int64_t am = s.idx(a, b, cc);
    const double w = G.vf(a, b, cc) / W.nov[am];
    v += w;
    x0 += w * (a + G.ce(0, a, b, cc));
    x1 += w * (b + G.ce(1, a, b, cc));
    x2 += w * (cc + G.ce(2, a, b, cc));
    for (int n = 0; n < NVAR; ++n) q[n] += w * (u(a, b, cc, n) + dt * W.divc[am + n * s.sn]);
  }
  W.vhat[at] = v;
  W.xhat[at] = x0 / v;
  W.xhat[at + s.sn] = x1 / v;
  W.xhat[at + 2 * s.sn] = x2 / v;
  for (int n = 0; n < NVAR; ++n) W.qhat[at + n * s.sn] = q[n] / v;
}

// Limited least-squares gradients of merged neighbourhoods on grow(bx,1).
__global__ void __launch_bounds__(kEB) k_srd_grad(Region r, EBWork W, EBG G) {
  int i, j, k;
  if (!region_cell(r, etid(), i, j, k)) return;
  const Space& s = W.s;
  const int64_t at = s.idx(i, j, k);
  const unsigned long long nw = W.nb[at];
  const int nn = nb_count(nw);
  if (nn < 2) return;
  const unsigned f = G.fl(i, j, k);
  const double* XH = W.xhat;
  const double xi0 = XH[at], xi1 = XH[at + s.sn], xi2 = XH[at + 2 * s.sn];
  double a00 = 0, a01 = 0, a02 = 0, a11 = 0, a12 = 0, a22 = 0;
  for (int kk = -1; kk <= 1; ++kk)
    for (int jj = -1; jj <= 1; ++jj)
      for (int ii = -1; ii <= 1; ++ii) {
        if ((ii == 0 && jj == 0 && kk == 0) || !f_conn(f, ii, jj, kk)) continue;
        const int64_t ak = s.idx(i + ii, j + jj, k + kk);
        if (nb_count(W.nb[ak]) == 0) continue;
        const double d0 = XH[ak] - xi0;
        const double d1 = XH[ak + s.sn] - xi1;
        const double d2 = XH[ak + 2 * s.sn] - xi2;
        a00 += d0 * d0; a01 += d0 * d1; a02 += d0 * d2;
        a11 += d1 * d1; a12 += d1 * d2; a22 += d2 * d2;
      }
  const double c00 = a11 * a22 - a12 * a12, c01 = a02 * a12 - a01 * a22,
               c02 = a01 * a12 - a02 * a11;
  const double det = a00 * c00 + a01 * c01 + a02 * c02;
  const double c11 = a00 * a22 - a02 * a02, c12 = a01 * a02 - a00 * a12,
               c22 = a00 * a11 - a01 * a01;
  for (int n = 0; n < NVAR; ++n) {
    double g0 = 0.0, g1 = 0.0, g2 = 0.0;
    if (fabs(det) > 1e-10) {
      const double* QH = W.qhat + n * s.sn;
      const double qi = QH[at];
      double b0 = 0, b1 = 0, b2 = 0;
      double qmin = qi, qmax = qi;
      for (int kk = -1; kk <= 1; ++kk)
        for (int jj = -1; jj <= 1; ++jj)
          for (int ii = -1; ii <= 1; ++ii) {
            if ((ii == 0 && jj == 0 && kk == 0) || !f_conn(f, ii, jj, kk)) continue;
            const int64_t ak = s.idx(i + ii, j + jj, k + kk);
            if (nb_count(W.nb[ak]) == 0) continue;
            const double d0 = XH[ak] - xi0;
            const double d1 = XH[ak + s.sn] - xi1;
            const double d2 = XH[ak + 2 * s.sn] - xi2;
            const double dq = QH[ak] - qi;
            b0 += d0 * dq; b1 += d1 * dq; b2 += d2 * dq;
            qmin = dmin(qmin, QH[ak]);
            qmax = dmax(qmax, QH[ak]);
          }
      g0 = (c00 * b0 + c01 * b1 + c02 * b2) / det;
      g1 = (c01 * b0 + c11 * b1 + c12 * b2) / det;
      g2 = (c02 * b0 + c12 * b1 + c22 * b2) / det;
      double alpha = 1.0;
      for (int c = 0; c < nn; ++c) {
        int di, dj, dk;
        off3(nb_off(nw, c), di, dj, dk);
        const int a = i + di, b = j + dj, cc = k + dk;
        const double v = g0 * (a + G.ce(0, a, b, cc) - xi0) + g1 * (b + G.ce(1, a, b, cc) - xi1) +
                         g2 * (cc + G.ce(2, a, b, cc) - xi2);
        if (v > 0.0) alpha = dmin(alpha, (qmax - qi) / v);
        else if (v < 0.0) alpha = dmin(alpha, (qmin - qi) / v);
      }
      g0 *= alpha;
      g1 *= alpha;
      g2 *= alpha;
    }
    W.grad[at + (3 * n) * s.sn] = g0;
    W.grad[at + (3 * n + 1) * s.sn] = g1;
    W.grad[at + (3 * n + 2) * s.sn] = g2;
  }
}

// The redistributed state of each cell of bx, gathered from the
// neighbourhoods that hold it (raster order), as a rate.
__global__ void __launch_bounds__(kEB) k_srd_final(Region r, EBWork W, EBG G, DFab u,
                                                    DtRef dtr, DFab dsdt) {
  int i, j, k;
  if (!region_cell(r, etid(), i, j, k)) return;
  if (f_covered(G.fl(i, j, k))) {
    for (int n = 0; n < NVAR; ++n) dsdt(i, j, k, n) = 0.0;
    return;
  }
  const Space& s = W.s;
  const double dt = dtr.get();
  double acc[NVAR];
  for (int n = 0; n < NVAR; ++n) acc[n] = 0.0;
  const double cx = i + G.ce(0, i, j, k), cy = j + G.ce(1, i, j, k), cz = k + G.ce(2, i, j, k);
  for (int kk = -1; kk <= 1; ++kk)
    for (int jj = -1; jj <= 1; ++jj)
      for (int ii = -1; ii <= 1; ++ii) {
        const int64_t aa = s.idx(i + ii, j + jj, k + kk);
        const unsigned long long nw = W.nb[aa];
        if (!nb_holds(nw, (1 - ii) + 3 * (1 - jj) + 9 * (1 - kk))) continue;
        if (nb_count(nw) < 2) {
          for (int n = 0; n < NVAR; ++n) acc[n] += W.qhat[aa + n * s.sn];
        } else {
          const double x0 = cx - W.xhat[aa];
          const double x1 = cy - W.xhat[aa + s.sn];
          const double x2 = cz - W.xhat[aa + 2 * s.sn];
          for (int n = 0; n < NVAR; ++n)
            acc[n] += W.qhat[aa + n * s.sn] + (W.grad[aa + (3 * n) * s.sn] * x0 +
                                               W.grad[aa + (3 * n + 1) * s.sn] * x1 +
                                               W.grad[aa + (3 * n + 2) * s.sn] * x2);
        }
      }
  const double nov = W.nov[s.idx(i, j, k)];
  for (int n = 0; n < NVAR; ++n) dsdt(i, j, k, n) = (acc[n] / nov - u(i, j, k, n)) / dt;
}

// One EB hydro evaluation of box bx: the launch geometry of K1-K8 and the
// workspace they share.  The workspace may be reused across evaluations of
// the same box: every intermediate a kernel reads is rewritten by an
// earlier kernel of the same evaluation or never written at all (covered
// cells' slopes, divergences and weights keep their first zero fill).
struct EBPlan {
  EBWork W;
  EBG G;
  KGeom g;
  KParams P;
  DBox db;
  int redist, wtype;
  bool mol;
  DtRef dt;                    // Godunov only
  Region rc, rsl, rd, rn, rf[3], ra[3];  // ctoprim, MOL slopes, divergence, div u nodes, faces
  Region r4, r3, r2, r1, r0;              // grow(bx, 4..0): redistribution
  DBox din;                                // inside the domain (non-periodic directions)
  int64_t ma;
  Region rq, rt, rf1[3];       // Godunov: q box, trace cells, first-pass faces
  Reg6E rf2;                   // Godunov: D|E faces
  int64_t mf1, mf2;
};

// The Space of bx: grown by ng (5 MOL, 6 Godunov: numGrow(), CAMR.H:465-472),
// one more high layer for faces.
inline Space eb_space(const int bx_lo[3], const int bx_hi[3], int ng) {
  Space s;
  for (int d = 0; d < 3; ++d) {
    s.lo[d] = bx_lo[d] - ng;
    s.n[d] = bx_hi[d] - bx_lo[d] + 1 + 2 * ng + 1;
  }
  s.sy = s.n[0];
  s.sz = s.sy * s.n[1];
  s.sn = s.sz * s.n[2];
  return s;
}

constexpr int kEBCommonComps = SQ_N + 3 * NVAR + 3 * 2 + 1 + NVAR + 1 + 2 * NVAR + 1;
constexpr int kEBSrdComps = 1 + 1 + 1 + 3 + NVAR + 3 * NVAR;
inline int eb_work_comps(bool mol, bool srd) {
  return kEBCommonComps + (mol ? 3 * SL_N : 6 * ES_N + 9 * FR_N) + (srd ? kEBSrdComps : 0);
}
// ghost cells: numGrow() (CAMR.H:465-479): 5 MOL / 6 Godunov with flux
// redistribution, one more with state redistribution
inline int eb_grow(bool mol, bool srd = false) { return (mol ? 5 : 6) + (srd ? 1 : 0); }

inline void eb_carve(EBWork& W, double* base, bool mol, bool srd = false) {
  double* ptr = base;
  auto take = [&](int nc) {
    double* r = ptr;
    ptr += size_t(nc) * W.s.sn;
    return r;
  };
  W.q = take(SQ_N);
  for (int d = 0; d < 3; ++d) {
    W.sl[d] = mol ? take(SL_N) : nullptr;
    W.sm[d] = mol ? nullptr : take(ES_N);
    W.sp[d] = mol ? nullptr : take(ES_N);
    W.f1[d] = mol ? nullptr : take(FR_N);
  }
  for (int c = 0; c < 6; ++c) W.f2[c] = mol ? nullptr : take(FR_N);
  for (int d = 0; d < 3; ++d) W.ft[d] = take(NVAR);
  for (int d = 0; d < 3; ++d) W.qf[d] = take(2);
  W.divu = take(1);
  W.divc = take(NVAR);
  W.wt = take(1);
  W.optmp = take(NVAR);
  W.delm = take(NVAR);
  W.wtinv = take(1);
  W.nb = srd ? reinterpret_cast<unsigned long long*>(take(1)) : nullptr;
  W.nov = srd ? take(1) : nullptr;
  W.vhat = srd ? take(1) : nullptr;
  W.xhat = srd ? take(3) : nullptr;
  W.qhat = srd ? take(NVAR) : nullptr;
  W.grad = srd ? take(3 * NVAR) : nullptr;
}

inline void eb_plan_init(EBPlan& E, const int bx_lo[3], const int bx_hi[3], const camr_geom& geom,
                         const camr_eb_geom& eb, const camr_hydro_params& p, int redist,
                         DtRef dt) {
  E.mol = p.do_mol != 0;
  E.dt = dt;
  const int e = (redist == 2) ? 1 : 0;  // state redistribution: one more layer
  E.W.s = eb_space(bx_lo, bx_hi, eb_grow(E.mol, e != 0));
  E.G.flag = eb.flag;
  E.G.vfrac = eb.vfrac;
  E.G.cent = eb.cent;
  for (int d = 0; d < 3; ++d) {
    E.G.ap[d] = eb.ap[d];
    E.G.fc[d] = eb.fc[d];
    E.G.lo[d] = eb.g_lo[d];
    E.G.n[d] = eb.g_hi[d] - eb.g_lo[d] + 1;
    E.g.lo[d] = bx_lo[d];
    E.g.hi[d] = bx_hi[d];
    E.g.dlo[d] = geom.dom_lo[d];
    E.g.dhi[d] = geom.dom_hi[d];
    E.g.bclo[d] = geom.bc_lo[d];
    E.g.bchi[d] = geom.bc_hi[d];
    E.g.dx[d] = geom.dx[d];
    E.db.lo[d] = geom.is_periodic[d] ? geom.dom_lo[d] - 2 : geom.dom_lo[d];
    E.db.hi[d] = geom.is_periodic[d] ? geom.dom_hi[d] + 2 : geom.dom_hi[d];
    E.din.lo[d] = geom.is_periodic[d] ? -(1 << 29) : geom.dom_lo[d];
    E.din.hi[d] = geom.is_periodic[d] ? (1 << 29) : geom.dom_hi[d];
  }
  E.P = make_kparams(p);
  E.redist = redist;
  E.wtype = p.eb_weights_type;
  auto reg = [&](int grow, int fdir, int tgrow) {
    int lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
      const int gr = (d == fdir) ? 0 : tgrow;
      lo[d] = bx_lo[d] - grow - gr;
      hi[d] = bx_hi[d] + grow + gr + (d == fdir ? 1 : 0);
    }
    return make_region(lo, hi);
  };
  // the divergence runs on grow(bx, 2+e) (bxg_i, CAMR_construct_hydro_source.cpp:146-152);
  // everything feeding it grows with it
  E.rc = reg(5 + e, -1, 0);
  E.rsl = reg(3 + e, -1, 0);
  E.rd = reg(2 + e, -1, 0);
  E.r4 = reg(4, -1, 0);
  E.r3 = reg(3, -1, 0);
  E.r2 = reg(2, -1, 0);
  E.r1 = reg(1, -1, 0);
  E.r0 = reg(0, -1, 0);
  E.ma = 0;
  for (int d = 0; d < 3; ++d) {
    E.rf[d] = reg(2 + e, d, 1);  // faces of grow(bx,2+e), transverse +1
    E.ra[d] = reg(3 + e, d, 0);  // faces of grow(bx,3+e)
    E.ma = E.ra[d].count() > E.ma ? E.ra[d].count() : E.ma;
  }
  // nodes of grow(bx,4+e) inside the domain grown by 16 in periodic directions
  int nlo[3], nhi[3];
  for (int d = 0; d < 3; ++d) {
    nlo[d] = bx_lo[d] - 4 - e;
    nhi[d] = bx_hi[d] + 5 + e;
    const int glo = geom.is_periodic[d] ? geom.dom_lo[d] - 16 : geom.dom_lo[d];
    const int ghi = geom.is_periodic[d] ? geom.dom_hi[d] + 1 + 16 : geom.dom_hi[d] + 1;
    nlo[d] = nlo[d] > glo ? nlo[d] : glo;
    nhi[d] = nhi[d] < ghi ? nhi[d] : ghi;
  }
  E.rn = make_region(nlo, nhi);
  // Godunov regions (Godunov_3D_eb.cpp, bx_to_fill = grow(bx,2)): q on
  // grow(bx,6), traces on grow(bx,4), first-pass E-faces [lo-3, hi+4] x
  // grow(bx,4), D|E faces [lo-3, hi+4] x E in grow(bx,3) x F in grow(bx,4)
  E.rq = reg(6 + e, -1, 0);
  E.rt = reg(4 + e, -1, 0);
  E.mf1 = E.mf2 = 0;
  for (int d = 0; d < 3; ++d) {
    int lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
      lo[a] = bx_lo[a] - (a == d ? 3 : 4) - e;
      hi[a] = bx_hi[a] + 4 + e;
    }
    E.rf1[d] = make_region(lo, hi);
    E.mf1 = E.rf1[d].count() > E.mf1 ? E.rf1[d].count() : E.mf1;
  }
  for (int D = 0; D < 3; ++D)
    for (int Ed = 0; Ed < 3; ++Ed) {
      if (Ed == D) continue;
      int lo[3], hi[3];
      for (int a = 0; a < 3; ++a) {
        const int gr = ((a == D) ? 3 : (a == Ed) ? 3 : 4) + e;
        lo[a] = bx_lo[a] - gr;
        hi[a] = bx_hi[a] + gr + (a == D ? 1 : 0);
      }
      Region& r = E.rf2.r[combo(D, Ed)];
      r = make_region(lo, hi);
      E.mf2 = r.count() > E.mf2 ? r.count() : E.mf2;
    }
}

// K1-K8 on the stream; fo[d].p may be null (no face-flux output).
// Returns the number of kernels issued.
inline int eb_issue(const EBPlan& E, const DFab& U, const DFab& dsdt, const DFab* fo,
                    cudaStream_t st) {
  int nk = 0;
  const EBWork& W = E.W;
  if (E.mol) {
    k_eb_ctoprim<<<eblk(E.rc.count()), kEB, 0, st>>>(E.rc, W, E.G, U, E.P, nullptr);
    k_eb_slope<<<dim3(eblk(E.rsl.count()), 3), kEB, 0, st>>>(E.rsl, W, E.G, E.P);
    nk += 2;
  } else {
    k_eb_ctoprim<<<eblk(E.rq.count()), kEB, 0, st>>>(E.rq, W, E.G, U, E.P, nullptr);
    k_ebc_trace<<<dim3(eblk(E.rt.count()), 3), kEB, 0, st>>>(E.rt, W, E.G, E.g, E.P, E.dt,
                                                             E.rq);
    k_ebc_flux1<<<dim3(eblk(E.mf1), 3), kEB, 0, st>>>(E.rf1[0], E.rf1[1], E.rf1[2], W, E.G,
                                                       E.g, E.P);
    k_ebc_flux2<<<dim3(eblk(E.mf2), 6), kEB, 0, st>>>(E.rf2, W, E.G, E.g, E.P, E.dt);
    nk += 4;
  }
  if (E.rn.count() > 0) {
    k_eb_divu<<<eblk(E.rn.count()), kEB, 0, st>>>(E.rn, W, E.G, E.g);
    ++nk;
  }
  if (E.mol) {
    k_eb_face<<<dim3(eblk(E.ma), 3), kEB, 0, st>>>(E.rf[0], E.rf[1], E.rf[2], E.ra[0], E.ra[1],
                                                    E.ra[2], W, E.G, E.g, E.P, U);
  } else {
    k_ebc_face<<<dim3(eblk(E.ma), 3), kEB, 0, st>>>(E.rf[0], E.rf[1], E.rf[2], E.ra[0],
                                                     E.ra[1], E.ra[2], W, E.G, E.g, E.P, U,
                                                     E.dt);
  }
  k_eb_div<<<eblk(E.rd.count()), kEB, 0, st>>>(E.rd, W, E.G, E.g, E.P, fo[0], fo[1], fo[2],
                                               E.wtype);
  nk += 2;
  if (E.redist == 2) {
    k_srd_nbhd<<<eblk(E.r4.count()), kEB, 0, st>>>(E.r4, W, E.G, E.din);
    k_srd_count<<<eblk(E.r3.count()), kEB, 0, st>>>(E.r3, W, E.G, E.din);
    k_srd_qhat<<<eblk(E.r2.count()), kEB, 0, st>>>(E.r2, W, E.G, U, E.dt);
    k_srd_grad<<<eblk(E.r1.count()), kEB, 0, st>>>(E.r1, W, E.G);
    k_srd_final<<<eblk(E.r0.count()), kEB, 0, st>>>(E.r0, W, E.G, U, E.dt, dsdt);
    return nk + 5;
  }
  if (E.redist) {
    k_eb_redist1<<<eblk(E.r1.count()), kEB, 0, st>>>(E.r1, W, E.G, E.db);
    ++nk;
  }
  k_eb_redist2<<<eblk(E.r0.count()), kEB, 0, st>>>(E.r0, W, E.G, E.db, E.g, dsdt, E.redist);
  ++nk;
  return nk;
}

// ---------------------------------------------------------------------------
// EB level: the level step of the single-level driver with the EB build's
// guards (Source/CAMR.cpp:877-891 normalize_species and :960-968
// enforce_min_density skip covered cells; reset_internal_energy runs where
// rho > 0, Utils/CAMR_reset_internal_e.H:36-38; computeTemp sets T = 0 first,
// Source/CAMR.cpp:1164-1168; the CFL minimum skips covered cells,
// Utils/Timestep.H:32-56).  The domain is one box with 5 ghost cells
// (CAMR::numGrow() with flux redistribution, Source/CAMR.H:455-479).

__device__ __forceinline__ void temp_eb(double* s, const KParams& P) {
  if (s[URHO] > 0.) {
    compute_temp(s, P);
  } else {
    s[UTEMP] = 0.0;
  }
}

__device__ __forceinline__ bool cov_at(const EBG& G, int i, int j, int k) {
  return f_covered(G.fl(i, j, k));
}

__global__ void __launch_bounds__(kBlk) k_ebl_est_dt(LGeom L, KParams P, EBG G, const double* S,
                                                      unsigned long long* bits) {
  int i, j, k;
  double v = DBL_MAX;
  if (valid_cell(L, tid(), i, j, k) && !cov_at(G, i, j, k)) {
    double s[NVAR];
    load_cell(S, L, L.idx(i, j, k), s);
    v = cell_dt(s, L, P);
  }
  block_min_dt(v, bits);
}

__global__ void __launch_bounds__(kBlk) k_ebl_clean_copy(LGeom L, KParams P, EBG G,
                                                          const double* S, double* out,
                                                          DevError* err, FloorList fl) {
  int i, j, k;
  if (!valid_cell(L, tid(), i, j, k)) return;
  const int64_t at = L.idx(i, j, k);
  double s[NVAR];
  load_cell(S, L, at, s);
  if (!cov_at(G, i, j, k)) {
    // below the floor: listed, k_floor_fixup redoes it in the reference's order
    if (s[URHO] < P.small_dens) floor_push(fl, at);
    enforce_min_density(s, S, L, P, i, j, k, err);
    normalize_species(s);
  }
  temp_eb(s, P);
  store_cell(out, L, at, s);
}

// expand_state with the EB guards (fill rules as k_expand's).
__global__ void __launch_bounds__(kBlk) k_ebl_expand(LGeom L, KParams P, EBG G,
                                                      const double* src, double* B,
                                                      DevError* err, FloorList fl) {
  int i, j, k;
  if (!padded_cell(L, tid(), i, j, k)) return;
  const int c[3] = {i, j, k};
  int img[3];
  bool physical = false;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    img[d] = c[d];
    if (c[d] < L.dlo[d] || c[d] > L.dhi[d]) {
      if (L.periodic[d]) {
        const int len = L.dhi[d] - L.dlo[d] + 1;
        img[d] = L.dlo[d] + (((c[d] - L.dlo[d]) % len) + len) % len;
      } else {
        physical = true;
      }
    }
  }
  double s[NVAR];
  if (!physical) {
    load_cell(src, L, L.idx(img[0], img[1], img[2]), s);
    if (!cov_at(G, img[0], img[1], img[2])) {
      // the valid cell itself (not a periodic ghost image) joins the list
      if (s[URHO] < P.small_dens && img[0] == i && img[1] == j && img[2] == k)
        floor_push(fl, L.idx(i, j, k));
      enforce_min_density(s, src, L, P, img[0], img[1], img[2], err);
      normalize_species(s);
    }
  } else {
#pragma unroll
    for (int n = 0; n < NVAR; ++n) {
      int id[3] = {img[0], img[1], img[2]};
      bool neg = false;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        if (L.periodic[d]) continue;
        if (id[d] < L.dlo[d]) {
          const int t = bc_kind(n, d, L.bclo[d]);
          if (t == 1 || t == 2) id[d] = L.dlo[d];
          else { id[d] = 2 * L.dlo[d] - id[d] - 1; if (t == 4) neg = !neg; }
        } else if (id[d] > L.dhi[d]) {
          const int t = bc_kind(n, d, L.bchi[d]);
          if (t == 1 || t == 2) id[d] = L.dhi[d];
          else { id[d] = 2 * L.dhi[d] - id[d] + 1; if (t == 4) neg = !neg; }
        }
      }
      const double v = src[L.idx(id[0], id[1], id[2]) + n * L.sn];
      s[n] = neg ? -v : v;
    }
  }
  temp_eb(s, P);
  store_cell(B, L, L.idx(i, j, k), s);
}

// MOL stage 1: S = Sborder (+ dt*src_old) + dt*k1.
__global__ void __launch_bounds__(kBlk) k_ebl_update1(LGeom L, KParams P, const double* dtp,
                                                       const double* B, const double* S_old,
                                                       const double* dsdt, double* S) {
  int i, j, k;
  if (!valid_cell(L, tid(), i, j, k)) return;
  const double dt = *dtp;
  const int64_t at = L.idx(i, j, k);
  double s[NVAR];
  load_cell(B, L, at, s);
  if (P.add_grav_src) {
    double src[NVAR];
#pragma unroll
    for (int n = 0; n < NVAR; ++n) src[n] = 0.0;
    src[UMZ] = P.const_grav * S_old[at + URHO * L.sn];
    src[UEDEN] = P.const_grav * S_old[at + UMZ * L.sn];
#pragma unroll
    for (int n = 0; n < NVAR; ++n) s[n] += dt * src[n];
  }
#pragma unroll
  for (int n = 0; n < NVAR; ++n) s[n] += dt * dsdt[at + n * L.sn];
  store_cell(S, L, at, s);
}

// clean_state of one cell inside the fused end of step.  The update
// kernels hand a cell below the density floor to k_floor_fixup before this
// point; one still below it here (or NaN) is reported.
__device__ __forceinline__ void clean_eb_cell(double* s, const KParams& P, bool cov, int i, int j,
                                              int k, DevError* err) {
  if (!cov) {
    if (!(s[URHO] >= P.small_dens)) report_error(err, s[URHO] == 0. ? 3 : 5, i, j, k);
    normalize_species(s);
  }
  temp_eb(s, P);
}

// The end of a level step on one cell: clean_state, the new-source
// correction (+ clean_state), post_timestep's clean_state; returns the
// cell's CFL dt (DBL_MAX on covered cells).
__device__ __forceinline__ double ebl_finish(double* s, const double* sold, const KParams& P,
                                             const LGeom& L, double dt, bool cov, int i, int j,
                                             int k, DevError* err) {
  clean_eb_cell(s, P, cov, i, j, k, err);
  if (P.add_grav_src) {
    double src[NVAR];
#pragma unroll
    for (int n = 0; n < NVAR; ++n) src[n] = 0.0;
    src[UMZ] = 0.5 * P.const_grav * (s[URHO] - sold[URHO]);
    src[UEDEN] = 0.5 * P.const_grav * (s[UMZ] - sold[UMZ]);
#pragma unroll
    for (int n = 0; n < NVAR; ++n) s[n] += dt * src[n];
    clean_eb_cell(s, P, cov, i, j, k, err);
  }
  clean_eb_cell(s, P, cov, i, j, k, err);
  return cov ? DBL_MAX : cell_dt(s, L, P);
}

// MOL stage 2: S = 0.5*Sborder2 + 0.5*S_old + 0.5*dt*k2, then the end of
// the step and the cell's CFL dt.
__global__ void __launch_bounds__(kBlk) k_ebl_update2(LGeom L, KParams P, EBG G,
                                                       const double* dtp, const double* B2,
                                                       const double* S_old, const double* dsdt,
                                                       double* S, unsigned long long* bits,
                                                       DevError* err, FloorList fl) {
  int i, j, k;
  double v = DBL_MAX;
  if (valid_cell(L, tid(), i, j, k)) {
    const double dt = *dtp;
    const int64_t at = L.idx(i, j, k);
    const bool cov = cov_at(G, i, j, k);
    double s[NVAR], sold[NVAR], b[NVAR];
    load_cell(B2, L, at, b);
    load_cell(S_old, L, at, sold);
#pragma unroll
    for (int n = 0; n < NVAR; ++n) s[n] = 0.5 * b[n] + 0.5 * sold[n];
#pragma unroll
    for (int n = 0; n < NVAR; ++n) s[n] += 0.5 * dt * dsdt[at + n * L.sn];
    // below the floor: the post-Saxpy state stays for k_floor_fixup
    if (!cov && s[URHO] < P.small_dens) floor_push(fl, at);
    else v = ebl_finish(s, sold, P, L, dt, cov, i, j, k, err);
    store_cell(S, L, at, s);
  }
  block_min_dt(v, bits);
}

// Godunov: S = Sborder (+ dt*src_old) + dt*dSdt, then the end of the step
// (CAMR_advance.cpp:101-121).
__global__ void __launch_bounds__(kBlk) k_ebl_update_ctu(LGeom L, KParams P, EBG G,
                                                          const double* dtp, const double* B,
                                                          const double* S_old,
                                                          const double* dsdt, double* S,
                                                          unsigned long long* bits,
                                                          DevError* err, FloorList fl) {
  int i, j, k;
  double v = DBL_MAX;
  if (valid_cell(L, tid(), i, j, k)) {
    const double dt = *dtp;
    const int64_t at = L.idx(i, j, k);
    const bool cov = cov_at(G, i, j, k);
    double s[NVAR], sold[NVAR];
    load_cell(B, L, at, s);
    load_cell(S_old, L, at, sold);
    if (P.add_grav_src) {
      double src[NVAR];
#pragma unroll
      for (int n = 0; n < NVAR; ++n) src[n] = 0.0;
      src[UMZ] = P.const_grav * sold[URHO];
      src[UEDEN] = P.const_grav * sold[UMZ];
#pragma unroll
      for (int n = 0; n < NVAR; ++n) s[n] += dt * src[n];
    }
#pragma unroll
    for (int n = 0; n < NVAR; ++n) s[n] += dt * dsdt[at + n * L.sn];
    if (!cov && s[URHO] < P.small_dens) floor_push(fl, at);
    else v = ebl_finish(s, sold, P, L, dt, cov, i, j, k, err);
    store_cell(S, L, at, s);
  }
  block_min_dt(v, bits);
}

// initData's epilogue with the EB guards: enforce_consistent_e where
// rho > 0 (Source/CAMR.cpp:910-939), then computeTemp.
__global__ void __launch_bounds__(kBlk) k_ebl_init_finalize(LGeom L, KParams P, double* S) {
  int i, j, k;
  if (!valid_cell(L, tid(), i, j, k)) return;
  const int64_t at = L.idx(i, j, k);
  double s[NVAR];
  load_cell(S, L, at, s);
  if (s[URHO] > 0.) {
    const double rhoInv = 1.0 / s[URHO];
    const double u = s[UMX] * rhoInv;
    const double v = s[UMY] * rhoInv;
    const double w = s[UMZ] * rhoInv;
    s[UEDEN] = s[UEINT] + 0.5 * s[URHO] * (u * u + v * v + w * w);
  }
  temp_eb(s, P);
  store_cell(S, L, at, s);
}

}  // namespace
}  // namespace camr

using namespace camr;

extern "C" camr_status camr_hydro_umdrv_eb(const int bx_lo[3], const int bx_hi[3],
                                           const camr_geom* geom, const camr_fab* uin,
                                           const camr_eb_geom* eb, camr_fab* dsdt,
                                           camr_fab* flx0, camr_fab* flx1, camr_fab* flx2,
                                           const camr_hydro_params* p, int redist, double dt,
                                           void* stream) {
  if (!bx_lo || !bx_hi || !geom || !uin || !eb || !dsdt || !flx0 || !flx1 || !flx2 || !p)
    return CAMR_ERR_INVALID;
  if (p->riemann_solver != 0) return CAMR_ERR_UNSUPPORTED;
  // Godunov with EB is PLM only (Source/CAMR.cpp:186-190)
  if (!p->do_mol && p->ppm_type != 0) return CAMR_ERR_INVALID;
  if (p->eb_weights_type < 0 || p->eb_weights_type > 3 || redist < 0 || redist > 2)
    return CAMR_ERR_INVALID;
  const int ng = eb_grow(p->do_mol != 0, redist == 2);
  for (int d = 0; d < 3; ++d) {
    if (bx_hi[d] < bx_lo[d]) return CAMR_ERR_INVALID;
    if (uin->lo[d] > bx_lo[d] - ng || uin->hi[d] < bx_hi[d] + ng) return CAMR_ERR_INVALID;
    if (eb->g_lo[d] > bx_lo[d] - ng || eb->g_hi[d] < bx_hi[d] + ng) return CAMR_ERR_INVALID;
  }
  if (!eb->flag || !eb->vfrac || !eb->ap[0] || !eb->ap[1] || !eb->ap[2] || !eb->fc[0] ||
      !eb->fc[1] || !eb->fc[2])
    return CAMR_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  EBPlan E;
  eb_plan_init(E, bx_lo, bx_hi, *geom, *eb, *p, redist, DtRef{dt, nullptr});
  const size_t bytes = size_t(eb_work_comps(E.mol, redist == 2)) * E.W.s.sn * sizeof(double);
  double* base = nullptr;
  if (cudaMallocAsync(reinterpret_cast<void**>(&base), bytes, st) != cudaSuccess)
    return CAMR_ERR_NOMEM;
  cudaError_t e = cudaMemsetAsync(base, 0, bytes, st);
  eb_carve(E.W, base, E.mol, redist == 2);
  // zero the output faces (covered cells leave theirs untouched)
  const DFab fo[3] = {make_dfab(*flx0), make_dfab(*flx1), make_dfab(*flx2)};
  int nk = 0;
  for (int d = 0; d < 3 && e == cudaSuccess; ++d) {
    int lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
      lo[a] = bx_lo[a];
      hi[a] = bx_hi[a] + (a == d ? 1 : 0);
    }
    const Region rf = make_region(lo, hi);
    k_eb_zero_faces<<<eblk(rf.count()), kEB, 0, st>>>(rf, fo[d]);
    ++nk;
  }
  if (e == cudaSuccess) nk += eb_issue(E, make_dfab(*uin), make_dfab(*dsdt), fo, st);
  count_launch(nk);
  if (e == cudaSuccess) e = cudaGetLastError();
  cudaError_t e2 = cudaFreeAsync(base, st);
  if (e != cudaSuccess) return cuda_status_of(e);
  return cuda_status_of(e2);
}

// ---------------------------------------------------------------------------
// EB level API.

struct camr_eb_level {
  camr_hydro_params hp;
  KParams P;
  camr_level_desc desc;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  LGeom L;
  int64_t ncell = 0, npad = 0;
  double *S = nullptr, *S_old = nullptr, *B = nullptr, *dsdt = nullptr;
  double *staging = nullptr, *fixed_dev = nullptr;
  double *dt_cur = nullptr, *dt_hist = nullptr;
  unsigned long long* bits = nullptr;
  int* nstep = nullptr;
  DevError* err = nullptr;
  FloorList floor;                // cells below the density floor of the current pass
  unsigned* flag = nullptr;
  double *vfrac = nullptr, *ap[3] = {nullptr, nullptr, nullptr}, *fc[3] = {nullptr, nullptr, nullptr};
  double* cent = nullptr;
  EBG G;                          // the level's geometry view (flags for the guards)
  std::vector<EBPlan> plans;      // cut boxes: EB hydro, one workspace each
  std::vector<double*> plan_work;
  camr_batch* regular = nullptr;  // regular boxes: the batched regular hydro
  double* regular_flx = nullptr;  // their face fluxes (scratch)
  int nbox_regular = 0, nbox_cut = 0, nbox_covered = 0;
  // side streams for the cut boxes: their launch sequences run concurrently
  // with each other and with the regular boxes' batch (fork/join by events,
  // captured into the step's graph as parallel branches)
  std::vector<cudaStream_t> side;
  cudaEvent_t ev_fork = nullptr;
  std::vector<cudaEvent_t> ev_join;
  int hist_cap = 1 << 16;
  int64_t steps_taken = 0;
  cudaGraphExec_t graph = nullptr;
  bool graph_ready = false;
  int64_t kernels_per_step = 0;
};

namespace {

DFab level_dfab(const LGeom& L, double* p) {
  DFab f;
  f.p = p;
  for (int d = 0; d < 3; ++d) f.lo[d] = L.plo[d];
  f.sy = L.sy;
  f.sz = L.sz;
  f.sn = L.sn;
  return f;
}

camr_fab level_fab(const LGeom& L, double* p) {
  camr_fab f;
  std::memset(&f, 0, sizeof(f));
  f.ptr = p;
  for (int d = 0; d < 3; ++d) {
    f.lo[d] = L.plo[d];
    f.hi[d] = L.plo[d] + L.pn[d] - 1;
  }
  f.jstride = L.sy;
  f.kstride = L.sz;
  f.nstride = L.sn;
  f.ncomp = NVAR;
  return f;
}

// construct_hydro_source of one stage (CAMR_construct_hydro_source.cpp:71-254
// in an EB build): src_to_fill = 0; per box: covered boxes nothing, boxes
// whose grow(bx,2) is all regular the regular hydro (batched), the others
// hydro_umdrv_eb.  Sborder is lev->B.
cudaError_t eb_hydro_stage(camr_eb_level* lev, cudaStream_t st, int* nk) {
  cudaError_t e = cudaMemsetAsync(lev->dsdt, 0, size_t(lev->L.sn) * NVAR * sizeof(double), st);
  const int nside = int(lev->side.size());
  if (nside && e == cudaSuccess) {
    e = cudaEventRecord(lev->ev_fork, st);
    for (cudaStream_t s2 : lev->side)
      if (e == cudaSuccess) e = cudaStreamWaitEvent(s2, lev->ev_fork, 0);
  }
  if (e != cudaSuccess) return e;
  const DFab none[3] = {level_dfab(lev->L, nullptr), level_dfab(lev->L, nullptr),
                        level_dfab(lev->L, nullptr)};
  const DFab U = level_dfab(lev->L, lev->B);
  const DFab ds = level_dfab(lev->L, lev->dsdt);
  for (size_t b = 0; b < lev->plans.size(); ++b)
    *nk += eb_issue(lev->plans[b], U, ds, none, nside ? lev->side[b % nside] : st);
  camr_status cs = CAMR_OK;
  if (lev->regular) cs = camr_batch_run(lev->regular, 0.0, lev->dt_cur, CAMR_BATCH_PERSISTENT, st);
  // the side streams join back whatever happened above, so that a capture
  // in progress ends with every branch joined
  for (int i = 0; i < nside; ++i) {
    const cudaError_t e1 = cudaEventRecord(lev->ev_join[i], lev->side[i]);
    const cudaError_t e2 = cudaStreamWaitEvent(st, lev->ev_join[i], 0);
    if (e == cudaSuccess) e = (e1 != cudaSuccess) ? e1 : e2;
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess && cs != CAMR_OK) e = cudaErrorLaunchFailure;
  return e;
}

cudaError_t eb_issue_step(camr_eb_level* lev, bool first, const double* fixed_dev) {
  const LGeom& L = lev->L;
  cudaStream_t st = lev->stream;
  const unsigned gv = grid_of(lev->ncell);
  const unsigned gp = grid_of(lev->npad);
  const EBG& G = lev->G;
  DtCtl c{lev->hp.cfl, lev->hp.max_dt, lev->hp.fixed_dt, lev->hp.initial_dt,
          lev->hp.init_shrink, lev->hp.change_max};
  int nk = 0;
  if (first) {
    k_reset_bits<<<1, 1, 0, st>>>(lev->bits);
    k_ebl_est_dt<<<gv, kBlk, 0, st>>>(L, lev->P, G, lev->S, lev->bits);
    nk += 2;
  }
  k_dt_next<<<1, 1, 0, st>>>(c, first ? 1 : 0, fixed_dev, lev->bits, lev->dt_cur, lev->dt_hist,
                             lev->nstep, lev->hist_cap);
  // Each cleaning pass lists the non-covered cells below the density floor
  // and a one-block fixup resets them in the reference's order (a no-op
  // launch when the list is empty).
  const FloorList& fl = lev->floor;
  FloorArgs fa{};
  fa.in = lev->S;
  fa.out = lev->S_old;
  k_ebl_clean_copy<<<gv, kBlk, 0, st>>>(L, lev->P, G, lev->S, lev->S_old, lev->err, fl);
  k_floor_fixup<FLOOR_CLEAN><<<1, 1024, kFloorSmem, st>>>(L, lev->P, fl, fa, lev->err);
  fa.in = lev->S_old;
  fa.out = lev->B;
  k_ebl_expand<<<gp, kBlk, 0, st>>>(L, lev->P, G, lev->S_old, lev->B, lev->err, fl);
  k_floor_fixup<FLOOR_EXPAND><<<1, 1024, kFloorSmem, st>>>(L, lev->P, fl, fa, lev->err);
  nk += 5;
  cudaError_t e = eb_hydro_stage(lev, st, &nk);
  if (e != cudaSuccess) return e;
  FloorArgs fu{};
  fu.out = lev->S;
  fu.B = lev->B;
  fu.S_old = lev->S_old;
  fu.dtp = lev->dt_cur;
  fu.bits = lev->bits;
  fu.post = 1;
  fu.dsdt = lev->dsdt;
  if (!lev->hp.do_mol) {
    k_ebl_update_ctu<<<gv, kBlk, 0, st>>>(L, lev->P, G, lev->dt_cur, lev->B, lev->S_old,
                                          lev->dsdt, lev->S, lev->bits, lev->err, fl);
    k_floor_fixup<FLOOR_DSDT_CTU><<<1, 1024, kFloorSmem, st>>>(L, lev->P, fl, fu, lev->err);
    count_launch(nk + 2);
    return cudaGetLastError();
  }
  k_ebl_update1<<<gv, kBlk, 0, st>>>(L, lev->P, lev->dt_cur, lev->B, lev->S_old, lev->dsdt,
                                     lev->S);
  // stage 2's Sborder reuses B (stage 1's is dead after the update)
  fa.in = lev->S;
  fa.out = lev->B;
  k_ebl_expand<<<gp, kBlk, 0, st>>>(L, lev->P, G, lev->S, lev->B, lev->err, fl);
  k_floor_fixup<FLOOR_EXPAND><<<1, 1024, kFloorSmem, st>>>(L, lev->P, fl, fa, lev->err);
  nk += 3;
  e = eb_hydro_stage(lev, st, &nk);
  if (e != cudaSuccess) return e;
  k_ebl_update2<<<gv, kBlk, 0, st>>>(L, lev->P, G, lev->dt_cur, lev->B, lev->S_old, lev->dsdt,
                                     lev->S, lev->bits, lev->err, fl);
  k_floor_fixup<FLOOR_DSDT_MOL2><<<1, 1024, kFloorSmem, st>>>(L, lev->P, fl, fu, lev->err);
  nk += 2;
  count_launch(nk);
  return cudaGetLastError();
}

// The level's boxes: the domain chopped by max_grid_size from the low end
// (the last box in a direction takes the remainder).
std::vector<std::array<int, 6>> level_boxes(const camr_geom& g, const int mgs[3]) {
  std::vector<std::array<int, 6>> out;
  int step[3];
  for (int d = 0; d < 3; ++d) {
    const int n = g.dom_hi[d] - g.dom_lo[d] + 1;
    step[d] = mgs[d] > 0 ? mgs[d] : n;
  }
  for (int k = g.dom_lo[2]; k <= g.dom_hi[2]; k += step[2])
    for (int j = g.dom_lo[1]; j <= g.dom_hi[1]; j += step[1])
      for (int i = g.dom_lo[0]; i <= g.dom_hi[0]; i += step[0])
        out.push_back({i, j, k, std::min(i + step[0] - 1, g.dom_hi[0]),
                       std::min(j + step[1] - 1, g.dom_hi[1]),
                       std::min(k + step[2] - 1, g.dom_hi[2])});
  return out;
}

}  // namespace

extern "C" {

camr_status camr_eb_level_create(const camr_level_desc* desc, const camr_eb_geom* eb,
                                 const camr_hydro_params* p, int redist, void* stream,
                                 camr_eb_level** out) {
  if (!desc || !eb || !p || !out) return CAMR_ERR_INVALID;
  *out = nullptr;
  if (p->riemann_solver != 0) return CAMR_ERR_UNSUPPORTED;
  if (floor_prepare() != cudaSuccess) return CAMR_ERR_CUDA;
  // Godunov with EB is PLM only (Source/CAMR.cpp:186-190); its predictor
  // sources are taken as zero, so no gravity with Godunov
  if (!p->do_mol && p->ppm_type != 0) return CAMR_ERR_INVALID;
  if (!p->do_mol && p->add_grav_src && p->const_grav != 0.0) return CAMR_ERR_UNSUPPORTED;
  if (p->eb_weights_type < 0 || p->eb_weights_type > 3 || redist < 0 || redist > 2)
    return CAMR_ERR_INVALID;
  const camr_geom& g = desc->geom;
  const int ng = eb_grow(p->do_mol != 0, redist == 2);
  for (int d = 0; d < 3; ++d) {
    if (g.dom_hi[d] < g.dom_lo[d]) return CAMR_ERR_INVALID;
    if (!g.is_periodic[d] && (g.bc_lo[d] == CAMR_BC_INTERIOR || g.bc_hi[d] == CAMR_BC_INTERIOR))
      return CAMR_ERR_INVALID;
    if (eb->g_lo[d] != g.dom_lo[d] - ng || eb->g_hi[d] != g.dom_hi[d] + ng)
      return CAMR_ERR_INVALID;
    if (desc->max_grid_size[d] < 0) return CAMR_ERR_INVALID;
  }
  if (!eb->flag || !eb->vfrac || !eb->ap[0] || !eb->ap[1] || !eb->ap[2] || !eb->fc[0] ||
      !eb->fc[1] || !eb->fc[2])
    return CAMR_ERR_INVALID;
  camr_eb_level* lev = new (std::nothrow) camr_eb_level();
  if (!lev) return CAMR_ERR_NOMEM;
  lev->hp = *p;
  lev->P = make_kparams(*p);
  lev->desc = *desc;
  lev->stream = static_cast<cudaStream_t>(stream);
  if (!lev->stream) {
    if (cudaStreamCreateWithFlags(&lev->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete lev;
      return CAMR_ERR_CUDA;
    }
    lev->own_stream = true;
  }
  LGeom& L = lev->L;
  for (int d = 0; d < 3; ++d) {
    L.dlo[d] = g.dom_lo[d];
    L.dhi[d] = g.dom_hi[d];
    L.plo[d] = g.dom_lo[d] - ng;
    L.pn[d] = g.dom_hi[d] - g.dom_lo[d] + 1 + 2 * ng;
    L.periodic[d] = g.is_periodic[d];
    L.bclo[d] = g.bc_lo[d];
    L.bchi[d] = g.bc_hi[d];
    L.dx[d] = g.dx[d];
    const int n = g.dom_hi[d] - g.dom_lo[d] + 1;
    L.boxsz[d] = desc->max_grid_size[d] > 0 ? desc->max_grid_size[d] : n;
  }
  L.sy = L.pn[0];
  L.sz = L.sy * L.pn[1];
  L.sn = L.sz * L.pn[2];
  lgeom_finish(L);
  lev->ncell = int64_t(g.dom_hi[0] - g.dom_lo[0] + 1) * (g.dom_hi[1] - g.dom_lo[1] + 1) *
               (g.dom_hi[2] - g.dom_lo[2] + 1);
  lev->npad = L.sn;
  const size_t state_bytes = size_t(L.sn) * NVAR * sizeof(double);
  int gn[3];
  for (int d = 0; d < 3; ++d) gn[d] = eb->g_hi[d] - eb->g_lo[d] + 1;
  const int64_t gc = int64_t(gn[0]) * gn[1] * gn[2];
  int64_t gf[3];
  for (int d = 0; d < 3; ++d) {
    gf[d] = 1;
    for (int a = 0; a < 3; ++a) gf[d] *= int64_t(gn[a] + (a == d));
  }
  cudaError_t e = cudaSuccess;
  auto alloc = [&](void** ptr, size_t b) {
    if (e == cudaSuccess) e = cudaMalloc(ptr, b);
    if (e == cudaSuccess) e = cudaMemsetAsync(*ptr, 0, b, lev->stream);
  };
  alloc(reinterpret_cast<void**>(&lev->S), state_bytes);
  alloc(reinterpret_cast<void**>(&lev->S_old), state_bytes);
  alloc(reinterpret_cast<void**>(&lev->B), state_bytes);
  alloc(reinterpret_cast<void**>(&lev->dsdt), state_bytes);
  alloc(reinterpret_cast<void**>(&lev->staging), size_t(lev->ncell) * NVAR * sizeof(double));
  alloc(reinterpret_cast<void**>(&lev->fixed_dev), sizeof(double));
  alloc(reinterpret_cast<void**>(&lev->dt_cur), sizeof(double));
  alloc(reinterpret_cast<void**>(&lev->dt_hist), sizeof(double) * lev->hist_cap);
  alloc(reinterpret_cast<void**>(&lev->bits), sizeof(unsigned long long));
  alloc(reinterpret_cast<void**>(&lev->nstep), sizeof(int));
  alloc(reinterpret_cast<void**>(&lev->err), sizeof(DevError));
  alloc(reinterpret_cast<void**>(&lev->floor.count), sizeof(int));
  alloc(reinterpret_cast<void**>(&lev->floor.cells), sizeof(int64_t) * kFloorCap);
  alloc(reinterpret_cast<void**>(&lev->floor.enforced), sizeof(double) * NVAR * kFloorCap);
  alloc(reinterpret_cast<void**>(&lev->floor.total), sizeof(unsigned long long));
  alloc(reinterpret_cast<void**>(&lev->flag), size_t(gc) * sizeof(unsigned));
  alloc(reinterpret_cast<void**>(&lev->vfrac), size_t(gc) * sizeof(double));
  if (eb->cent) alloc(reinterpret_cast<void**>(&lev->cent), size_t(3 * gc) * sizeof(double));
  for (int d = 0; d < 3; ++d) {
    alloc(reinterpret_cast<void**>(&lev->ap[d]), size_t(gf[d]) * sizeof(double));
    alloc(reinterpret_cast<void**>(&lev->fc[d]), size_t(2 * gf[d]) * sizeof(double));
  }
  // the geometry is copied into the level (device or host source)
  auto copy = [&](void* dst, const void* src, size_t b) {
    if (e == cudaSuccess) e = cudaMemcpyAsync(dst, src, b, cudaMemcpyDefault, lev->stream);
  };
  copy(lev->flag, eb->flag, size_t(gc) * sizeof(unsigned));
  copy(lev->vfrac, eb->vfrac, size_t(gc) * sizeof(double));
  if (eb->cent) copy(lev->cent, eb->cent, size_t(3 * gc) * sizeof(double));
  for (int d = 0; d < 3; ++d) {
    copy(lev->ap[d], eb->ap[d], size_t(gf[d]) * sizeof(double));
    copy(lev->fc[d], eb->fc[d], size_t(2 * gf[d]) * sizeof(double));
  }
  std::vector<unsigned> hflag(static_cast<size_t>(gc));
  if (e == cudaSuccess) e = cudaStreamSynchronize(lev->stream);
  if (e == cudaSuccess)
    e = cudaMemcpy(hflag.data(), lev->flag, size_t(gc) * sizeof(unsigned), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    camr_eb_level_destroy(lev);
    return e == cudaErrorMemoryAllocation ? CAMR_ERR_NOMEM : cuda_status_of(e);
  }
  camr_eb_geom own = *eb;
  own.flag = lev->flag;
  own.vfrac = lev->vfrac;
  for (int d = 0; d < 3; ++d) {
    own.ap[d] = lev->ap[d];
    own.fc[d] = lev->fc[d];
    own.cent = lev->cent;
    lev->G.lo[d] = eb->g_lo[d];
    lev->G.n[d] = gn[d];
    lev->G.ap[d] = lev->ap[d];
    lev->G.fc[d] = lev->fc[d];
  }
  lev->G.flag = lev->flag;
  lev->G.cent = lev->cent;
  lev->G.vfrac = lev->vfrac;
  // classify the boxes (CAMR_construct_hydro_source.cpp:76-78, :150-153)
  auto typ = [&](int i, int j, int k) {
    return hflag[size_t((i - eb->g_lo[0]) +
                        int64_t(gn[0]) * ((j - eb->g_lo[1]) + int64_t(gn[1]) * (k - eb->g_lo[2])))] &
           3u;
  };
  std::vector<camr_box_task> reg_tasks;
  std::vector<std::array<int, 6>> cut_boxes;
  for (const auto& b : level_boxes(g, desc->max_grid_size)) {
    bool all_cov = true;
    for (int k = b[2]; k <= b[5] && all_cov; ++k)
      for (int j = b[1]; j <= b[4] && all_cov; ++j)
        for (int i = b[0]; i <= b[3]; ++i)
          if (typ(i, j, k) != 3u) {
            all_cov = false;
            break;
          }
    if (all_cov) {
      lev->nbox_covered++;
      continue;
    }
    bool all_reg = true;
    // grow(box, 2), or 3 with state redistribution (CAMR_construct_hydro_source.cpp:146-153)
    const int gb = (redist == 2) ? 3 : 2;
    for (int k = b[2] - gb; k <= b[5] + gb && all_reg; ++k)
      for (int j = b[1] - gb; j <= b[4] + gb && all_reg; ++j)
        for (int i = b[0] - gb; i <= b[3] + gb; ++i)
          if (typ(i, j, k) != 0u) {
            all_reg = false;
            break;
          }
    if (all_reg) {
      camr_box_task t;
      std::memset(&t, 0, sizeof(t));
      for (int d = 0; d < 3; ++d) {
        t.lo[d] = b[d];
        t.hi[d] = b[3 + d];
      }
      t.uin = level_fab(L, lev->B);
      t.dsdt = level_fab(L, lev->dsdt);
      reg_tasks.push_back(t);
    } else {
      cut_boxes.push_back(b);
    }
  }
  lev->nbox_regular = int(reg_tasks.size());
  lev->nbox_cut = int(cut_boxes.size());
  // regular boxes: face-flux scratch, then the batch plan
  if (!reg_tasks.empty()) {
    size_t per = 0;
    std::vector<size_t> off(reg_tasks.size());
    for (size_t b = 0; b < reg_tasks.size(); ++b) {
      off[b] = per;
      for (int d = 0; d < 3; ++d) {
        int64_t n = NVAR;
        for (int a = 0; a < 3; ++a) n *= (reg_tasks[b].hi[a] - reg_tasks[b].lo[a] + 1 + (a == d));
        per += size_t(n);
      }
    }
    alloc(reinterpret_cast<void**>(&lev->regular_flx), per * sizeof(double));
    for (size_t b = 0; b < reg_tasks.size() && e == cudaSuccess; ++b) {
      double* ptr = lev->regular_flx + off[b];
      camr_box_task& t = reg_tasks[b];
      for (int d = 0; d < 3; ++d) {
        camr_fab& f = t.flx[d];
        f.ptr = ptr;
        int ext[3];
        for (int a = 0; a < 3; ++a) {
          f.lo[a] = t.lo[a];
          f.hi[a] = t.hi[a] + (a == d);
          ext[a] = f.hi[a] - f.lo[a] + 1;
        }
        f.jstride = ext[0];
        f.kstride = int64_t(ext[0]) * ext[1];
        f.nstride = f.kstride * ext[2];
        f.ncomp = NVAR;
        ptr += f.nstride * NVAR;
      }
    }
    if (e == cudaSuccess) {
      const camr_status cs = batch_create_eb(int(reg_tasks.size()), reg_tasks.data(), &g, p,
                                             lev->stream, lev->flag, eb->g_lo, gn,
                                             &lev->regular);
      if (cs != CAMR_OK) {
        camr_eb_level_destroy(lev);
        return cs;
      }
    }
  }
  // cut boxes: one EB plan and workspace each, spread over side streams
  // at the device's greatest priority: a cut box's chain of small launches
  // is the critical path of a hydro stage, so its blocks go first whenever
  // the regular boxes' blocks retire
  const int nside = int(std::min<size_t>(cut_boxes.size(), 8));
  int prio_least = 0, prio_greatest = 0;
  if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest);
  if (e == cudaSuccess && nside > 0) e = cudaEventCreateWithFlags(&lev->ev_fork, cudaEventDisableTiming);
  for (int i = 0; i < nside && e == cudaSuccess; ++i) {
    cudaStream_t s2;
    cudaEvent_t ej;
    e = cudaStreamCreateWithPriority(&s2, cudaStreamNonBlocking, prio_greatest);
    if (e != cudaSuccess) break;
    lev->side.push_back(s2);
    e = cudaEventCreateWithFlags(&ej, cudaEventDisableTiming);
    if (e != cudaSuccess) break;
    lev->ev_join.push_back(ej);
  }
  for (const auto& b : cut_boxes) {
    const int lo[3] = {b[0], b[1], b[2]}, hi[3] = {b[3], b[4], b[5]};
    EBPlan E;
    eb_plan_init(E, lo, hi, g, own, *p, redist, DtRef{0.0, lev->dt_cur});
    double* w = nullptr;
    alloc(reinterpret_cast<void**>(&w),
          size_t(eb_work_comps(E.mol, redist == 2)) * E.W.s.sn * sizeof(double));
    if (e != cudaSuccess) break;
    lev->plan_work.push_back(w);
    eb_carve(E.W, w, E.mol, redist == 2);
    lev->plans.push_back(E);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(lev->stream);
  if (e != cudaSuccess) {
    camr_eb_level_destroy(lev);
    return e == cudaErrorMemoryAllocation ? CAMR_ERR_NOMEM : cuda_status_of(e);
  }
  *out = lev;
  return CAMR_OK;
}

camr_status camr_eb_level_destroy(camr_eb_level* lev) {
  if (!lev) return CAMR_ERR_INVALID;
  if (lev->graph_ready) cudaGraphExecDestroy(lev->graph);
  if (lev->regular) camr_batch_destroy(lev->regular);
  void* ptrs[] = {lev->S,       lev->S_old,   lev->B,      lev->dsdt,       lev->staging,
                  lev->fixed_dev, lev->dt_cur, lev->dt_hist, lev->bits,     lev->nstep,
                  lev->err,     lev->flag,    lev->vfrac,  lev->ap[0],      lev->ap[1],
                  lev->ap[2],   lev->fc[0],   lev->fc[1],  lev->fc[2],      lev->regular_flx,
                  lev->cent,    lev->floor.count, lev->floor.cells, lev->floor.enforced,
                  lev->floor.total};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  for (double* w : lev->plan_work)
    if (w) cudaFree(w);
  for (cudaEvent_t ev : lev->ev_join) cudaEventDestroy(ev);
  if (lev->ev_fork) cudaEventDestroy(lev->ev_fork);
  for (cudaStream_t s2 : lev->side) cudaStreamDestroy(s2);
  if (lev->own_stream) cudaStreamDestroy(lev->stream);
  delete lev;
  return CAMR_OK;
}

camr_status camr_eb_level_set_state(camr_eb_level* lev, const double* state, int host) {
  if (!lev || !state) return CAMR_ERR_INVALID;
  const size_t bytes = size_t(lev->ncell) * NVAR * sizeof(double);
  cudaError_t e = cudaMemcpyAsync(lev->staging, state, bytes,
                                  host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                                  lev->stream);
  if (e != cudaSuccess) return cuda_status_of(e);
  k_pack<<<grid_of(lev->ncell), kBlk, 0, lev->stream>>>(lev->L, lev->S, lev->staging, 0);
  count_launch();
  lev->steps_taken = 0;
  return cuda_status_of(cudaGetLastError());
}

camr_status camr_eb_level_get_state(camr_eb_level* lev, double* state, int host) {
  if (!lev || !state) return CAMR_ERR_INVALID;
  k_pack<<<grid_of(lev->ncell), kBlk, 0, lev->stream>>>(lev->L, lev->S, lev->staging, 1);
  count_launch();
  const size_t bytes = size_t(lev->ncell) * NVAR * sizeof(double);
  cudaError_t e = cudaMemcpyAsync(state, lev->staging, bytes,
                                  host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                                  lev->stream);
  if (e == cudaSuccess && host) e = cudaStreamSynchronize(lev->stream);
  return cuda_status_of(e);
}

camr_status camr_eb_level_init_finalize(camr_eb_level* lev) {
  if (!lev) return CAMR_ERR_INVALID;
  k_ebl_init_finalize<<<grid_of(lev->ncell), kBlk, 0, lev->stream>>>(lev->L, lev->P, lev->S);
  count_launch();
  return cuda_status_of(cudaGetLastError());
}

camr_status camr_eb_level_advance(camr_eb_level* lev, int nsteps, const double* fixed_dts) {
  if (!lev || nsteps < 0) return CAMR_ERR_INVALID;
  for (int s = 0; s < nsteps; ++s) {
    const bool first = lev->steps_taken == 0;
    const double* fixed_dev = nullptr;
    cudaError_t e;
    if (fixed_dts) {
      e = cudaMemcpyAsync(lev->fixed_dev, &fixed_dts[s], sizeof(double), cudaMemcpyHostToDevice,
                          lev->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(lev->stream);
      if (e != cudaSuccess) return cuda_status_of(e);
      fixed_dev = lev->fixed_dev;
    }
    if (!first && !fixed_dts && lev->desc.use_graph) {
      if (!lev->graph_ready) {
        cudaGraph_t gr;
        e = cudaStreamBeginCapture(lev->stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return cuda_status_of(e);
        const int64_t before = launches_now();
        const cudaError_t e1 = eb_issue_step(lev, false, nullptr);
        lev->kernels_per_step = launches_now() - before;
        launches_sub(lev->kernels_per_step);
        e = cudaStreamEndCapture(lev->stream, &gr);
        if (e1 != cudaSuccess) return cuda_status_of(e1);
        if (e != cudaSuccess) return cuda_status_of(e);
        e = cudaGraphInstantiate(&lev->graph, gr, 0);
        cudaGraphDestroy(gr);
        if (e != cudaSuccess) return cuda_status_of(e);
        lev->graph_ready = true;
      }
      e = cudaGraphLaunch(lev->graph, lev->stream);
      count_launch(int(lev->kernels_per_step));
    } else {
      e = eb_issue_step(lev, first, fixed_dev);
    }
    if (e != cudaSuccess) return cuda_status_of(e);
    lev->steps_taken++;
  }
  return CAMR_OK;
}

camr_status camr_eb_level_dts(camr_eb_level* lev, double* dts, int n, int* nsteps) {
  if (!lev || (n > 0 && !dts)) return CAMR_ERR_INVALID;
  int taken = 0;
  cudaError_t e = cudaMemcpyAsync(&taken, lev->nstep, sizeof(int), cudaMemcpyDeviceToHost,
                                  lev->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(lev->stream);
  if (e != cudaSuccess) return cuda_status_of(e);
  if (nsteps) *nsteps = taken;
  const int m = taken < n ? taken : n;
  const int cap = m < lev->hist_cap ? m : lev->hist_cap;
  if (cap > 0) {
    e = cudaMemcpyAsync(dts, lev->dt_hist, sizeof(double) * cap, cudaMemcpyDeviceToHost,
                        lev->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(lev->stream);
  }
  return cuda_status_of(e);
}

camr_status camr_eb_level_autotune(camr_eb_level* lev) {
  if (!lev) return CAMR_ERR_INVALID;
  if (!lev->regular) return CAMR_OK;
  double dt = 0.0;
  cudaError_t e = cudaMemcpyAsync(&dt, lev->dt_cur, sizeof(double), cudaMemcpyDeviceToHost,
                                  lev->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(lev->stream);
  if (e != cudaSuccess) return cuda_status_of(e);
  constexpr int NS = BS_COUNT;
  int chunk[3][NS];
  unsigned grid[3][NS];
  // candidate 2: the untuned shapes
  camr_status cs = camr_batch_tuning(lev->regular, chunk[2], grid[2], NS);
  if (cs == CAMR_OK) cs = camr_batch_autotune(lev->regular, dt, lev->stream);
  if (cs == CAMR_OK) cs = camr_batch_tuning(lev->regular, chunk[0], grid[0], NS);
  if (cs != CAMR_OK) return cs;
  // candidate 0: each stage timed alone; candidate 1: the same cells per
  // block with one block per work unit, which leaves SMs free for the cut
  // boxes' launches on the side streams as blocks retire
  for (int s = 0; s < NS; ++s) {
    chunk[1][s] = chunk[0][s];
    grid[1][s] = 0;
  }
  // a whole hydro stage (dSdt zeroed, then regular and cut boxes) only reads
  // Sborder, so it can be repeated; it is timed as a captured graph, the
  // form the level's steps take: one untimed launch, the best of three
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  int best_c = 0;
  for (int c = 0; c < 3 && e == cudaSuccess; ++c) {
    camr_batch_set_tuning(lev->regular, chunk[c], grid[c], NS);
    int nk = 0;
    cudaGraph_t gr = nullptr;
    cudaGraphExec_t gx = nullptr;
    e = cudaStreamBeginCapture(lev->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) break;
    const int64_t before = launches_now();
    const cudaError_t e1c = eb_hydro_stage(lev, lev->stream, &nk);
    launches_sub(launches_now() - before);
    e = cudaStreamEndCapture(lev->stream, &gr);
    if (e == cudaSuccess) e = e1c;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&gx, gr, 0);
    if (gr) cudaGraphDestroy(gr);
    if (e == cudaSuccess) e = cudaGraphLaunch(gx, lev->stream);
    for (int r = 0; r < 3 && e == cudaSuccess; ++r) {
      cudaEventRecord(e0, lev->stream);
      e = cudaGraphLaunch(gx, lev->stream);
      cudaEventRecord(e1, lev->stream);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (e == cudaSuccess && ms < best) {
        best = ms;
        best_c = c;
      }
    }
    if (gx) cudaGraphExecDestroy(gx);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  camr_batch_set_tuning(lev->regular, chunk[best_c], grid[best_c], NS);
  if (e != cudaSuccess) return cuda_status_of(e);
  // a captured step holds the old launch shapes
  if (lev->graph_ready) {
    cudaGraphExecDestroy(lev->graph);
    lev->graph_ready = false;
  }
  return cs;
}

camr_status camr_eb_level_boxes(camr_eb_level* lev, int* regular, int* cut, int* covered) {
  if (!lev) return CAMR_ERR_INVALID;
  if (regular) *regular = lev->nbox_regular;
  if (cut) *cut = lev->nbox_cut;
  if (covered) *covered = lev->nbox_covered;
  return CAMR_OK;
}

int64_t camr_eb_level_kernels_per_step(camr_eb_level* lev) {
  return lev ? lev->kernels_per_step : 0;
}

camr_status camr_eb_level_stream(camr_eb_level* lev, void** stream) {
  if (!lev || !stream) return CAMR_ERR_INVALID;
  *stream = lev->stream;
  return CAMR_OK;
}

camr_status camr_eb_level_floor_resets(camr_eb_level* lev, int64_t* cells) {
  if (!lev || !cells) return CAMR_ERR_INVALID;
  unsigned long long h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, lev->floor.total, sizeof(h), cudaMemcpyDeviceToHost,
                                  lev->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(lev->stream);
  if (e != cudaSuccess) return cuda_status_of(e);
  *cells = int64_t(h);
  return CAMR_OK;
}

camr_status camr_eb_level_get_error(camr_eb_level* lev, camr_error_info* info) {
  if (!lev || !info) return CAMR_ERR_INVALID;
  DevError h{};
  cudaError_t e = cudaMemcpyAsync(&h, lev->err, sizeof(h), cudaMemcpyDeviceToHost, lev->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(lev->err, 0, sizeof(DevError), lev->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(lev->stream);
  if (e != cudaSuccess) return cuda_status_of(e);
  info->code = h.code;
  info->i = h.i;
  info->j = h.j;
  info->k = h.k;
  return h.code ? CAMR_ERR_NUMERIC : CAMR_OK;
}

}  // extern "C"
