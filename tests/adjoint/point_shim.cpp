// CPU build of the adjoint's pointwise forward/VJP functions for the finite-
// difference tests (tests/test_adjoint_point.py).  Flat double arrays in and
// out; layouts documented per function.
#include "../../camr_b200/csrc/adjoint_point.cuh"

using namespace camr::adj;

static Par par_of(const double* p) {
  Par P;
  P.gamma = p[0]; P.small = p[1]; P.small_dens = p[2]; P.small_pres = p[3]; P.smallu = p[4];
  P.small_num = p[5]; P.difmag = p[6]; P.eta1 = p[7]; P.eta2 = p[8]; P.small_temp = p[9];
  P.dual_energy_update_E_from_e = 1;
  return P;
}

// Face input vector (62 doubles): qL[11] qR[11] sL[8] sR[8] dv[4] uL[10] uR[10]
static void unpack_face(const double* x, FaceIn& in) {
  int o = 0;
  for (int n = 0; n < NQ; ++n) in.qL[n] = x[o++];
  for (int n = 0; n < NQ; ++n) in.qR[n] = x[o++];
  for (int n = 0; n < NS; ++n) in.sL[n] = x[o++];
  for (int n = 0; n < NS; ++n) in.sR[n] = x[o++];
  for (int n = 0; n < 4; ++n) in.dv[n] = x[o++];
  for (int n = 0; n < NV; ++n) in.uL[n] = x[o++];
  for (int n = 0; n < NV; ++n) in.uR[n] = x[o++];
}
static void pack_face(const FaceIn& in, double* x) {
  int o = 0;
  for (int n = 0; n < NQ; ++n) x[o++] = in.qL[n];
  for (int n = 0; n < NQ; ++n) x[o++] = in.qR[n];
  for (int n = 0; n < NS; ++n) x[o++] = in.sL[n];
  for (int n = 0; n < NS; ++n) x[o++] = in.sR[n];
  for (int n = 0; n < 4; ++n) x[o++] = in.dv[n];
  for (int n = 0; n < NV; ++n) x[o++] = in.uL[n];
  for (int n = 0; n < NV; ++n) x[o++] = in.uR[n];
}

template <int d>
static void face_f(const double* p, const double* x, double* y) {
  Par P = par_of(p);
  FaceIn in;
  unpack_face(x, in);
  FaceTape t;
  FaceOut o;
  face_forward<d>(in, p[10], p[11], P, t, o);
  for (int n = 0; n < NV; ++n) y[n] = o.f[n];
  y[10] = o.qpres;
  y[11] = o.qun;
}
template <int d>
static void face_b(const double* p, const double* x, const double* by, double* bx) {
  Par P = par_of(p);
  FaceIn in, bin;
  unpack_face(x, in);
  double z[62] = {0};
  unpack_face(z, bin);
  FaceTape t;
  FaceOut o, bo;
  face_forward<d>(in, p[10], p[11], P, t, o);
  for (int n = 0; n < NV; ++n) bo.f[n] = by[n];
  bo.qpres = by[10];
  bo.qun = by[11];
  face_vjp<d>(in, p[10], p[11], P, t, bo, bin);
  pack_face(bin, bx);
}

template <int d>
static void slope_f(const double* p, const double* x, double* y) {
  Par P = par_of(p);
  SlopeTape t;
  slope_fwd<d>(x, x + NQ, x + 2 * NQ, P, t, y);
}
template <int d>
static void slope_b(const double* p, const double* x, const double* by, double* bx) {
  Par P = par_of(p);
  SlopeTape t;
  double y[NS];
  slope_fwd<d>(x, x + NQ, x + 2 * NQ, P, t, y);
  for (int n = 0; n < 3 * NQ; ++n) bx[n] = 0.0;
  slope_vjp<d>(x, x + NQ, x + 2 * NQ, P, t, by, bx, bx + NQ, bx + 2 * NQ);
}

extern "C" {
void adj_face_fwd(int d, const double* p, const double* x, double* y) {
  if (d == 0) face_f<0>(p, x, y);
  else if (d == 1) face_f<1>(p, x, y);
  else face_f<2>(p, x, y);
}
void adj_face_vjp(int d, const double* p, const double* x, const double* by, double* bx) {
  if (d == 0) face_b<0>(p, x, by, bx);
  else if (d == 1) face_b<1>(p, x, by, bx);
  else face_b<2>(p, x, by, bx);
}
// x: qm[11] q0[11] qp[11]; y: 8 slopes
void adj_slope_fwd(int d, const double* p, const double* x, double* y) {
  if (d == 0) slope_f<0>(p, x, y);
  else if (d == 1) slope_f<1>(p, x, y);
  else slope_f<2>(p, x, y);
}
void adj_slope_vjp(int d, const double* p, const double* x, const double* by, double* bx) {
  if (d == 0) slope_b<0>(p, x, by, bx);
  else if (d == 1) slope_b<1>(p, x, by, bx);
  else slope_b<2>(p, x, by, bx);
}
// x: U[10]; y: q[11]
void adj_ctoprim_fwd(const double* p, const double* x, double* y) {
  Par P = par_of(p);
  bool br;
  ctoprim_fwd(x, P, y, br);
}
void adj_ctoprim_vjp(const double* p, const double* x, const double* by, double* bx) {
  Par P = par_of(p);
  for (int n = 0; n < NV; ++n) bx[n] = 0.0;
  ctoprim_vjp(x, P, by, bx);
}
// x: U[10]; y: clean(U)[10]
void adj_clean_fwd(const double* p, const double* x, double* y) {
  Par P = par_of(p);
  CleanTape t;
  clean_fwd(x, P, t, y);
}
void adj_clean_vjp(const double* p, const double* x, const double* by, double* bx) {
  Par P = par_of(p);
  for (int n = 0; n < NV; ++n) bx[n] = 0.0;
  clean_vjp(x, P, by, bx);
}
}
