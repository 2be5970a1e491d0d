// Restated single-level driver around the per-box hydro (test oracle).
//
// Restates, line by line, the parts of CAMR and of the AMReX calls it makes
// that sit between the per-box hydro call and a whole time step:
//   CAMR::CAMR_advance            Source/CAMR_advance.cpp:38-164
//   CAMR::expand_state/clean_state Source/CAMR.cpp:1243-1262
//   enforce_min_density           Source/CAMR.cpp:941-1045
//   normalize_species             Source/CAMR.cpp:866-908
//   computeTemp                   Source/CAMR.cpp:1141-1185
//   reset_internal_energy         Source/Utils/CAMR_reset_internal_e.H:13-129
//   gravity sources               Source/GravitySrc.cpp:4-121
//   estTimeStep / computeNewDt    Source/CAMR.cpp:490-635, Source/Utils/Timestep.H:18-61
//   enforce_consistent_e          Source/CAMR.cpp:910-939
//   FillPatch physical BCs        Source/Utils/CAMR_setup.cpp:19-21 (BC tables),
//                                 AMReX foextrap / reflect_even / reflect_odd
// The per-box hydro comes from orc_hydro_box, which each oracle library
// implements (restated or the reference's own code).
#include <omp.h>

#include <cstring>

#include "oracle_common.hpp"

namespace orc {
namespace {

struct Grid {
  Box3 dom;
  int n[3];
  long long ncell;
  std::vector<Box3> tiles;  // hydro tiles (boxes cut by tile_size)
  std::vector<Box3> boxes;
};

Grid make_grid(const orc_level& L) {
  Grid g;
  for (int d = 0; d < 3; ++d) {
    g.dom.lo[d] = L.dom_lo[d];
    g.dom.hi[d] = L.dom_hi[d];
    g.n[d] = L.dom_hi[d] - L.dom_lo[d] + 1;
  }
  g.ncell = 1LL * g.n[0] * g.n[1] * g.n[2];
  int mgs[3];
  for (int d = 0; d < 3; ++d) mgs[d] = L.max_grid_size[d] > 0 ? L.max_grid_size[d] : g.n[d];
  for (int k = g.dom.lo[2]; k <= g.dom.hi[2]; k += mgs[2])
    for (int j = g.dom.lo[1]; j <= g.dom.hi[1]; j += mgs[1])
      for (int i = g.dom.lo[0]; i <= g.dom.hi[0]; i += mgs[0]) {
        Box3 b;
        b.lo[0] = i; b.lo[1] = j; b.lo[2] = k;
        b.hi[0] = std::min(i + mgs[0] - 1, g.dom.hi[0]);
        b.hi[1] = std::min(j + mgs[1] - 1, g.dom.hi[1]);
        b.hi[2] = std::min(k + mgs[2] - 1, g.dom.hi[2]);
        g.boxes.push_back(b);
      }
  for (const Box3& b : g.boxes) {
    int ts[3];
    for (int d = 0; d < 3; ++d) ts[d] = L.tile_size[d] > 0 ? L.tile_size[d] : (b.hi[d] - b.lo[d] + 1);
    for (int k = b.lo[2]; k <= b.hi[2]; k += ts[2])
      for (int j = b.lo[1]; j <= b.hi[1]; j += ts[1])
        for (int i = b.lo[0]; i <= b.hi[0]; i += ts[0]) {
          Box3 t;
          t.lo[0] = i; t.lo[1] = j; t.lo[2] = k;
          t.hi[0] = std::min(i + ts[0] - 1, b.hi[0]);
          t.hi[1] = std::min(j + ts[1] - 1, b.hi[1]);
          t.hi[2] = std::min(k + ts[2] - 1, b.hi[2]);
          g.tiles.push_back(t);
        }
  }
  return g;
}

int nthreads_of(const orc_level& L) { return L.nthreads > 0 ? L.nthreads : 1; }

// computeTemp body on one cell: reset_internal_energy then T.
void reset_internal_e(const Eos& eos, const orc_params& p, const Fab& S, int i, int j, int k) {
  const double rho = S(i, j, k, URHO);
  const double rhoInv = 1.0 / rho;
  const double Up = S(i, j, k, UMX) * rhoInv;
  const double Vp = S(i, j, k, UMY) * rhoInv;
  const double Wp = S(i, j, k, UMZ) * rhoInv;
  const double ke = 0.5 * (Up * Up + Vp * Vp + Wp * Wp);
  const double eden = S(i, j, k, UEDEN) * rhoInv;
  double massfrac[NSPEC];
  for (int s = 0; s < NSPEC; ++s) massfrac[s] = S(i, j, k, s + UFS) * rhoInv;
  double e_out = 0.;
  double small_e = 0.;
  const double small_T = p.small_temp;
  if (p.allow_small_energy == 0) {
    small_e = eos.rty2e(small_T, massfrac);
    if (eden < small_e) {
      if (S(i, j, k, UEINT) * rhoInv < small_e) {
        const double T = std::max(S(i, j, k, UTEMP), small_T);
        e_out = eos.rty2e(T, massfrac);
        S(i, j, k, UEINT) = rho * e_out;
      }
      S(i, j, k, UEDEN) = S(i, j, k, UEINT) + rho * ke;
    } else {
      const double rho_eint = S(i, j, k, UEDEN) - S(i, j, k, URHO) * ke;
      if (rho_eint > 0. && rho_eint / S(i, j, k, UEDEN) > p.dual_energy_eta2) {
        S(i, j, k, UEINT) = rho_eint;
      }
      if (S(i, j, k, UEINT) * rhoInv < small_e) {
        const double T = std::max(S(i, j, k, UTEMP), small_T);
        e_out = eos.rty2e(T, massfrac);
        if (p.dual_energy_update_E_from_e == 1) {
          S(i, j, k, UEDEN) += (rho * e_out - S(i, j, k, UEINT));
        }
        S(i, j, k, UEINT) = S(i, j, k, URHO) * e_out;
      }
    }
  } else if (p.allow_negative_energy == 0) {
    if (S(i, j, k, UEDEN) < 0.) {
      if (S(i, j, k, UEINT) < 0.) {
        e_out = eos.rty2e(small_T, massfrac);
        S(i, j, k, UEINT) = rho * e_out;
      }
      S(i, j, k, UEDEN) = S(i, j, k, UEINT) + rho * ke;
    } else {
      const double rho_eint = S(i, j, k, UEDEN) - rho * ke;
      if (rho_eint > 0. && rho_eint / S(i, j, k, UEDEN) > p.dual_energy_eta2) {
        S(i, j, k, UEINT) = rho_eint;
      } else if (S(i, j, k, UEINT) > 0 && p.dual_energy_update_E_from_e == 1) {
        S(i, j, k, UEDEN) = S(i, j, k, UEINT) + rho * ke;
      } else if (S(i, j, k, UEINT) <= 0.) {
        e_out = eos.rty2e(small_T, massfrac);
        S(i, j, k, UEINT) = rho * e_out;
        if (p.dual_energy_update_E_from_e == 1) {
          S(i, j, k, UEDEN) += (rho * e_out - S(i, j, k, UEINT));
        }
      }
    }
  } else {
    S(i, j, k, UEINT) = S(i, j, k, UEDEN) - rho * ke;
  }
}

void compute_temp_cell(const Eos& eos, const orc_params& p, const Fab& S, int i, int j, int k) {
  reset_internal_e(eos, p, S, i, j, k);
  const double rhoInv = 1.0 / S(i, j, k, URHO);
  const double e = S(i, j, k, UEINT) * rhoInv;
  S(i, j, k, UTEMP) = eos.ey2t(e);
}

void normalize_species_cell(const Fab& S, int i, int j, int k) {
  double sum = 0.;
  for (int s = 0; s < NSPEC; ++s) {
    S(i, j, k, UFS + s) = std::max(std::min(S(i, j, k, URHO), S(i, j, k, UFS + s)), 0.0);
    sum += S(i, j, k, UFS + s);
  }
  if (S(i, j, k, URHO) > 0.) {
    sum /= S(i, j, k, URHO);
    for (int s = 0; s < NSPEC; ++s) S(i, j, k, UFS + s) /= sum;
  }
}

// enforce_min_density on one tile, in the CPU loop order of the reference.
long enforce_min_density_tile(const Eos& eos, const orc_params& p, const Fab& S, const Box3& t) {
  long nerr = 0;
  for_box(t, [&](int i, int j, int k) {
    if (S(i, j, k, URHO) == 0.) {
      ++nerr;  // amrex::Error in the reference
    } else if (S(i, j, k, URHO) < p.small_dens) {
      double max_dens = S(i, j, k, URHO);
      int is = i, js = j, ks = k;
      for (int kk = -1; kk <= 1; kk++)
        for (int jj = -1; jj <= 1; jj++)
          for (int ii = -1; ii <= 1; ii++) {
            if (i + ii >= t.lo[0] && j + jj >= t.lo[1] && k + kk >= t.lo[2] &&
                i + ii <= t.hi[0] && j + jj <= t.hi[1] && k + kk <= t.hi[2]) {
              if (S(i + ii, j + jj, k + kk, URHO) > max_dens) {
                is = i + ii; js = j + jj; ks = k + kk;
                max_dens = S(is, js, ks, URHO);
              }
            }
          }
      if (max_dens < p.small_dens) {
        double massfrac[NSPEC];
        for (int s = 0; s < NSPEC; ++s) massfrac[s] = S(i, j, k, UFS + s) / S(i, j, k, URHO);
        const double small_e = eos.rty2e(p.small_temp, massfrac);
        S(i, j, k, URHO) = p.small_dens;
        S(i, j, k, UTEMP) = p.small_temp;
        S(i, j, k, UMX) = 0.;
        S(i, j, k, UMY) = 0.;
        S(i, j, k, UMZ) = 0.;
        S(i, j, k, UEINT) = p.small_dens * small_e;
        S(i, j, k, UEDEN) = S(i, j, k, UEINT);
      } else {
        for (int n = 0; n < NVAR; ++n) S(i, j, k, n) = S(is, js, ks, n);
      }
    }
  });
  return nerr;
}

template <class F>
void par_cells(const Grid& g, int nth, F&& f) {
  const int nz = g.n[2];
#pragma omp parallel for num_threads(nth) schedule(static)
  for (int kk = 0; kk < nz; ++kk) {
    const int k = g.dom.lo[2] + kk;
    for (int j = g.dom.lo[1]; j <= g.dom.hi[1]; ++j)
      for (int i = g.dom.lo[0]; i <= g.dom.hi[0]; ++i) f(i, j, k);
  }
}

// clean_state on valid cells only (a MultiFab without ghost cells).
long clean_state_valid(const Eos& eos, const orc_params& p, const orc_level& L, const Grid& g,
                       const Fab& S) {
  long nerr = 0;
  const int nth = nthreads_of(L);
  const int nt = int(g.tiles.size());
#pragma omp parallel for num_threads(nth) reduction(+ : nerr) schedule(dynamic)
  for (int t = 0; t < nt; ++t) nerr += enforce_min_density_tile(eos, p, S, g.tiles[t]);
  par_cells(g, nth, [&](int i, int j, int k) { normalize_species_cell(S, i, j, k); });
  par_cells(g, nth, [&](int i, int j, int k) { compute_temp_cell(eos, p, S, i, j, k); });
  return nerr;
}

int bc_type_of(int n, int dir, int phys) {
  // Source/Utils/CAMR_setup.cpp:19-21: 0 int_dir, 1 ext_dir, 2 foextrap,
  // 3 reflect_even, 4 reflect_odd (local encoding).
  static const int scalar_bc[] = {0, 1, 2, 3, 3, 3};
  static const int norm_vel_bc[] = {0, 1, 2, 4, 4, 4};
  static const int tang_vel_bc[] = {0, 1, 2, 3, 3, 4};
  if (n == UMX || n == UMY || n == UMZ) {
    const int vdir = n - UMX;
    return (vdir == dir) ? norm_vel_bc[phys] : tang_vel_bc[phys];
  }
  return scalar_bc[phys];
}

// Value of the physical-boundary ghost cell (i,j,k), component n, from the
// valid data S (FillPatch's periodic copy then the BC function).
double physbc_value(const orc_level& L, const Grid& g, const Fab& S, int i, int j, int k, int n) {
  int idx[3] = {i, j, k};
  double sign = 1.0;
  for (int d = 0; d < 3; ++d) {
    const int lo = g.dom.lo[d], hi = g.dom.hi[d];
    if (L.is_periodic[d]) {
      const int len = hi - lo + 1;
      idx[d] = lo + (((idx[d] - lo) % len) + len) % len;
      continue;
    }
    if (idx[d] < lo) {
      const int t = bc_type_of(n, d, L.bc_lo[d]);
      if (t == 1 || t == 2) idx[d] = lo;
      else { idx[d] = 2 * lo - idx[d] - 1; if (t == 4) sign = -sign; }
    } else if (idx[d] > hi) {
      const int t = bc_type_of(n, d, L.bc_hi[d]);
      if (t == 1 || t == 2) idx[d] = hi;
      else { idx[d] = 2 * hi - idx[d] + 1; if (t == 4) sign = -sign; }
    }
  }
  const double v = S(idx[0], idx[1], idx[2], n);
  return sign < 0 ? -v : v;
}

// FillPatch(S) into B (domain grown by ng) followed by clean_state(B).
long expand_state(const Eos& eos, const orc_params& p, const orc_level& L, const Grid& g,
                  const Fab& S, const Fab& B) {
  const int nth = nthreads_of(L);
  // FillPatch copy of the valid region.
  par_cells(g, nth, [&](int i, int j, int k) {
    for (int n = 0; n < NVAR; ++n) B(i, j, k, n) = S(i, j, k, n);
  });
  // clean_state(B): enforce_min_density and normalize_species on valid cells.
  long nerr = 0;
  const int nt = int(g.tiles.size());
#pragma omp parallel for num_threads(nth) reduction(+ : nerr) schedule(dynamic)
  for (int t = 0; t < nt; ++t) nerr += enforce_min_density_tile(eos, p, B, g.tiles[t]);
  par_cells(g, nth, [&](int i, int j, int k) { normalize_species_cell(B, i, j, k); });
  // Ghost cells: FillBoundary for those inside the periodic extension of the
  // domain, FillPatch's physical-BC values (from S) for the rest.
  const int nz = B.hi[2] - B.lo[2] + 1;
#pragma omp parallel for num_threads(nth) schedule(static)
  for (int kk = 0; kk < nz; ++kk) {
    const int k = B.lo[2] + kk;
    for (int j = B.lo[1]; j <= B.hi[1]; ++j)
      for (int i = B.lo[0]; i <= B.hi[0]; ++i) {
        const int idx[3] = {i, j, k};
        bool inside = true, physical = false;
        int img[3];
        for (int d = 0; d < 3; ++d) {
          img[d] = idx[d];
          if (idx[d] < g.dom.lo[d] || idx[d] > g.dom.hi[d]) {
            inside = false;
            if (L.is_periodic[d]) {
              const int len = g.n[d];
              img[d] = g.dom.lo[d] + (((idx[d] - g.dom.lo[d]) % len) + len) % len;
            } else {
              physical = true;
            }
          }
        }
        if (inside) continue;
        if (!physical) {
          for (int n = 0; n < NVAR; ++n) B(i, j, k, n) = B(img[0], img[1], img[2], n);
        } else {
          for (int n = 0; n < NVAR; ++n) B(i, j, k, n) = physbc_value(L, g, S, i, j, k, n);
        }
      }
  }
  // computeTemp(B, ng) on every cell.
#pragma omp parallel for num_threads(nth) schedule(static)
  for (int kk = 0; kk < nz; ++kk) {
    const int k = B.lo[2] + kk;
    for (int j = B.lo[1]; j <= B.hi[1]; ++j)
      for (int i = B.lo[0]; i <= B.hi[0]; ++i) compute_temp_cell(eos, p, B, i, j, k);
  }
  return nerr;
}

// construct_hydro_source over all tiles: dsdt = 0, then each tile's hydro.
// Coarse side of a two-level flux register (restating AMReX YAFluxRegister
// for refinement ratio 2): per coarse cell, its fine-box id (-1 if not
// covered), the coarse cells outside the fine region that share a face
// with it ("boundary cells"), and the accumulated correction d.
struct FluxReg {
  Fab d;                    // NVAR comps on the coarse domain (CrseAdd sums)
  Fab cfp;                  // NVAR comps on the coarse domain (FineAdd sums)
  std::vector<int> cmap;    // coarse cell -> fine box id or -1
  std::vector<char> bnd;    // coarse cell is a coarse-fine boundary cell
  int lo[3], n[3];
  int periodic[3];
  int cell(int i, int j, int k) const {
    int c[3] = {i, j, k};
    for (int d = 0; d < 3; ++d) {
      int v = c[d] - lo[d];
      if (periodic[d]) v = ((v % n[d]) + n[d]) % n[d];
      else if (v < 0 || v >= n[d]) return -1;
      c[d] = v;
    }
    return c[0] + n[0] * (c[1] + n[1] * c[2]);
  }
  int box_at(int i, int j, int k) const {
    const int c = cell(i, j, k);
    return c < 0 ? -1 : cmap[c];
  }
};

// YAFluxRegister::CrseAdd on one tile: for every coarse-fine boundary cell
// of the tile, remove the coarse flux through each face it shares with a
// fine-covered cell (faces in the order x-, x+, y-, y+, z-, z+), scaled by
// dt/vol (the fluxes are area-weighted).
void crse_add(FluxReg& fr, const Box3& bx, const Fab* f, double dtdx) {
  for_box(bx, [&](int i, int j, int k) {
    const int c = fr.cell(i, j, k);
    if (c < 0 || !fr.bnd[c]) return;
    const int e[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int d = 0; d < 3; ++d) {
      if (fr.box_at(i - e[d][0], j - e[d][1], k - e[d][2]) >= 0) {
        for (int n = 0; n < NVAR; ++n) fr.d(i, j, k, n) -= dtdx * f[d](i, j, k, n);
      }
      if (fr.box_at(i + e[d][0], j + e[d][1], k + e[d][2]) >= 0) {
        for (int n = 0; n < NVAR; ++n)
          fr.d(i, j, k, n) += dtdx * f[d](i + e[d][0], j + e[d][1], k + e[d][2], n);
      }
    }
  });
}

long hydro_level(const orc_params& p, const orc_level& L, const Grid& g, const Fab& B,
                 const Fab* src, const Fab& dsdt, double dt, FluxReg* fr = nullptr,
                 double fr_dtdx = 0.0) {
  const int nth = nthreads_of(L);
  par_cells(g, nth, [&](int i, int j, int k) {
    for (int n = 0; n < NVAR; ++n) dsdt(i, j, k, n) = 0.0;
  });
  long nerr = 0;
  const int nt = int(g.tiles.size());
#pragma omp parallel for num_threads(nth) reduction(+ : nerr) schedule(dynamic)
  for (int t = 0; t < nt; ++t) {
    const Box3& bx = g.tiles[t];
    std::vector<double> f[3];
    for (int d = 0; d < 3; ++d) {
      const Box3 fb = faces(bx, d);
      f[d].resize(size_t(fb.hi[0] - fb.lo[0] + 1) * (fb.hi[1] - fb.lo[1] + 1) *
                  (fb.hi[2] - fb.lo[2] + 1) * NVAR);
    }
    nerr += orc_hydro_box(&p, bx.lo, bx.hi, L.dom_lo, L.dom_hi, L.bc_lo, L.bc_hi, B.p, B.lo,
                          B.hi, src ? src->p : nullptr, dsdt.p, dsdt.lo, dsdt.hi,
                          f[0].data(), f[1].data(), f[2].data(), L.dx, dt);
    if (fr) {
      Fab ff[3];
      for (int d = 0; d < 3; ++d) {
        const Box3 fb = faces(bx, d);
        ff[d].view(f[d].data(), fb.lo, fb.hi, NVAR);
      }
      crse_add(*fr, bx, ff, fr_dtdx);
    }
  }
  return nerr;
}

double est_dt(const Eos& eos, const orc_params& p, const orc_level& L, const Grid& g,
              const Fab& S) {
  if (p.fixed_dt > 0.0) return p.fixed_dt;
  double estdt = p.max_dt;
  const double max_dt_over_cfl = p.max_dt / p.cfl;
  double estdt_hydro = max_dt_over_cfl;
  double dt = std::numeric_limits<double>::max();
  const int nth = nthreads_of(L);
  const int nz = g.n[2];
#pragma omp parallel for num_threads(nth) reduction(min : dt) schedule(static)
  for (int kk = 0; kk < nz; ++kk) {
    const int k = g.dom.lo[2] + kk;
    for (int j = g.dom.lo[1]; j <= g.dom.hi[1]; ++j)
      for (int i = g.dom.lo[0]; i <= g.dom.hi[0]; ++i) {
        const double rho = S(i, j, k, URHO);
        const double rhoInv = 1.0 / rho;
        const double eint = S(i, j, k, UEINT) / rho;
        const double pres = eos.rey2p(rho, eint);
        const double gam = eos.gamma;
        const double c = std::sqrt(gam * pres / rho);
        const double ux = S(i, j, k, UMX) * rhoInv;
        const double dt1 = L.dx[0] / (c + std::fabs(ux));
        dt = std::min(dt, dt1);
        const double uy = S(i, j, k, UMY) * rhoInv;
        const double dt2 = L.dx[1] / (c + std::fabs(uy));
        dt = std::min(dt, dt2);
        const double uz = S(i, j, k, UMZ) * rhoInv;
        const double dt3 = L.dx[2] / (c + std::fabs(uz));
        dt = std::min(dt, dt3);
      }
  }
  estdt_hydro = std::min(estdt_hydro, dt);
  estdt_hydro *= p.cfl;
  if (estdt_hydro < estdt) estdt = estdt_hydro;
  return estdt;
}

// Gravity source terms (GravitySrc.cpp:36-121): old uses S_old, the
// correction uses S_new and S_old; both begin from setVal(0).
void grav_old(const orc_params& p, const Grid& g, int nth, const Fab& S_old, const Fab& src) {
  par_cells(g, nth, [&](int i, int j, int k) {
    for (int n = 0; n < NVAR; ++n) src(i, j, k, n) = 0.0;
    src(i, j, k, UMZ) = p.const_grav * S_old(i, j, k, URHO);
    src(i, j, k, UEDEN) = p.const_grav * S_old(i, j, k, UMZ);
  });
}

void grav_new(const orc_params& p, const Grid& g, int nth, const Fab& S_old, const Fab& S_new,
              const Fab& src) {
  par_cells(g, nth, [&](int i, int j, int k) {
    for (int n = 0; n < NVAR; ++n) src(i, j, k, n) = 0.0;
    src(i, j, k, UMZ) = 0.5 * p.const_grav * (S_new(i, j, k, URHO) - S_old(i, j, k, URHO));
    src(i, j, k, UEDEN) = 0.5 * p.const_grav * (S_new(i, j, k, UMZ) - S_old(i, j, k, UMZ));
  });
}

struct Work {
  Fab S_old, B, B2, dsdt, dsdt2, src_old, src_new, sfh;
};

// One CAMR::advance + post_timestep on the state S (valid cells), in place.
long advance_one(const Eos& eos, const orc_params& p, const orc_level& L, const Grid& g,
                 const Fab& S, Work& w, double dt, FluxReg* fr = nullptr, bool post = true) {
  // CrseAdd scale of one construct_hydro_source call: fac_for_reflux*dt/vol
  // (CAMR_construct_hydro_source.cpp:24, :245-247).
  const double vol = L.dx[0] * L.dx[1] * L.dx[2];
  const double fr_dtdx = ((p.do_mol ? 0.5 : 1.0) * dt) / vol;
  const int nth = nthreads_of(L);
  long nerr = 0;
  // swapTimeLevels: S_old <- S; clean_state(S_old).
  par_cells(g, nth, [&](int i, int j, int k) {
    for (int n = 0; n < NVAR; ++n) w.S_old(i, j, k, n) = S(i, j, k, n);
  });
  nerr += clean_state_valid(eos, p, L, g, w.S_old);
  nerr += expand_state(eos, p, L, g, w.S_old, w.B);
  // S_new = Sborder (valid).
  par_cells(g, nth, [&](int i, int j, int k) {
    for (int n = 0; n < NVAR; ++n) S(i, j, k, n) = w.B(i, j, k, n);
  });
  if (p.add_grav_src) {
    grav_old(p, g, nth, w.S_old, w.src_old);
    par_cells(g, nth, [&](int i, int j, int k) {
      for (int n = 0; n < NVAR; ++n) S(i, j, k, n) += dt * w.src_old(i, j, k, n);
    });
  }
  if (p.do_mol) {
    nerr += hydro_level(p, L, g, w.B, nullptr, w.dsdt, dt, fr, fr_dtdx);
    par_cells(g, nth, [&](int i, int j, int k) {
      for (int n = 0; n < NVAR; ++n) S(i, j, k, n) += dt * w.dsdt(i, j, k, n);
    });
    nerr += expand_state(eos, p, L, g, S, w.B2);
    nerr += hydro_level(p, L, g, w.B2, nullptr, w.dsdt2, dt, fr, fr_dtdx);
    par_cells(g, nth, [&](int i, int j, int k) {
      for (int n = 0; n < NVAR; ++n) {
        S(i, j, k, n) = 0.5 * w.B2(i, j, k, n) + 0.5 * w.S_old(i, j, k, n);
      }
    });
    par_cells(g, nth, [&](int i, int j, int k) {
      for (int n = 0; n < NVAR; ++n) S(i, j, k, n) += 0.5 * dt * w.dsdt2(i, j, k, n);
    });
  } else {
    // sources_for_hydro = 0 + 1.0*old sources on valid cells, FillBoundary
    // on periodic/interior ghosts, zero on physical-boundary ghosts.
    const Fab& sf = w.sfh;
    for (auto& v : w.sfh.own) v = 0.0;
    if (p.add_grav_src) {
      par_cells(g, nth, [&](int i, int j, int k) {
        for (int n = 0; n < NVAR; ++n) sf(i, j, k, n) += 1.0 * w.src_old(i, j, k, n);
      });
      for_box(Box3{{sf.lo[0], sf.lo[1], sf.lo[2]}, {sf.hi[0], sf.hi[1], sf.hi[2]}},
              [&](int i, int j, int k) {
                const int idx[3] = {i, j, k};
                bool inside = true, physical = false;
                int img[3];
                for (int d = 0; d < 3; ++d) {
                  img[d] = idx[d];
                  if (idx[d] < g.dom.lo[d] || idx[d] > g.dom.hi[d]) {
                    inside = false;
                    if (L.is_periodic[d]) {
                      img[d] = g.dom.lo[d] + (((idx[d] - g.dom.lo[d]) % g.n[d]) + g.n[d]) % g.n[d];
                    } else {
                      physical = true;
                    }
                  }
                }
                if (inside || physical) return;
                for (int n = 0; n < NVAR; ++n) sf(i, j, k, n) = sf(img[0], img[1], img[2], n);
              });
    }
    nerr += hydro_level(p, L, g, w.B, &w.sfh, w.dsdt, dt, fr, fr_dtdx);
    par_cells(g, nth, [&](int i, int j, int k) {
      for (int n = 0; n < NVAR; ++n) S(i, j, k, n) += dt * w.dsdt(i, j, k, n);
    });
  }
  nerr += clean_state_valid(eos, p, L, g, S);
  if (p.add_grav_src) {
    grav_new(p, g, nth, w.S_old, S, w.src_new);
    par_cells(g, nth, [&](int i, int j, int k) {
      for (int n = 0; n < NVAR; ++n) S(i, j, k, n) += dt * w.src_new(i, j, k, n);
    });
    nerr += clean_state_valid(eos, p, L, g, S);
  }
  // CAMR::post_timestep: clean_state(S_new).
  if (post) nerr += clean_state_valid(eos, p, L, g, S);
  return nerr;
}

void alloc_work(const Grid& g, Work& w) {
  const Box3 b4 = grow(g.dom, 4);
  w.S_old.alloc(g.dom.lo, g.dom.hi, NVAR);
  w.B.alloc(b4.lo, b4.hi, NVAR);
  w.B2.alloc(b4.lo, b4.hi, NVAR);
  w.dsdt.alloc(g.dom.lo, g.dom.hi, NVAR);
  w.dsdt2.alloc(g.dom.lo, g.dom.hi, NVAR);
  w.src_old.alloc(g.dom.lo, g.dom.hi, NVAR);
  w.src_new.alloc(g.dom.lo, g.dom.hi, NVAR);
  w.sfh.alloc(b4.lo, b4.hi, NVAR);
}


// ===========================================================================
// Two-level AMR with subcycling (refinement ratio 2), restating AMReX's
// Amr::timeStep / FillPatchTwoLevels / YAFluxRegister / average_down as
// CAMR drives them (Source/CAMR_advance.cpp:38-164, Source/CAMR.cpp:566-635,
// :679-718, :803-851, :1048-1066; Source/Hydro/CAMR_construct_hydro_source.cpp:243-254).
// AMReX itself is absent, so these steps follow its documented algorithms;
// the order of a few floating-point sums (flux-register contributions to one
// coarse cell) is this file's choice.  Periodic domains only.

constexpr int RR = 2;  // refinement ratio

struct Fine {
  std::vector<Box3> boxes;
  orc_level L;
  std::vector<Fab> S, S_old, B, B2, dsdt, dsdt2, sfh;
  std::vector<std::vector<double>> fbuf[3];
  std::vector<Fab> F[3];  // face fluxes of the last hydro call
};

inline int wrap(int v, int lo, int n) { return lo + (((v - lo) % n) + n) % n; }

FluxReg make_fluxreg(const Grid& gc, const orc_level& Lc, const std::vector<Box3>& fboxes) {
  FluxReg fr;
  for (int d = 0; d < 3; ++d) {
    fr.lo[d] = gc.dom.lo[d];
    fr.n[d] = gc.n[d];
    fr.periodic[d] = Lc.is_periodic[d];
  }
  const size_t nc = size_t(gc.ncell);
  fr.cmap.assign(nc, -1);
  fr.bnd.assign(nc, 0);
  for (int b = 0; b < int(fboxes.size()); ++b) {
    Box3 cb;
    for (int d = 0; d < 3; ++d) {
      cb.lo[d] = fboxes[b].lo[d] / RR;
      cb.hi[d] = fboxes[b].hi[d] / RR;
    }
    for_box(cb, [&](int i, int j, int k) { fr.cmap[fr.cell(i, j, k)] = b; });
  }
  for_box(gc.dom, [&](int i, int j, int k) {
    const int c = fr.cell(i, j, k);
    if (fr.cmap[c] >= 0) return;
    const int e[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int d = 0; d < 3; ++d)
      if (fr.box_at(i - e[d][0], j - e[d][1], k - e[d][2]) >= 0 ||
          fr.box_at(i + e[d][0], j + e[d][1], k + e[d][2]) >= 0)
        fr.bnd[c] = 1;
  });
  fr.d.alloc(gc.dom.lo, gc.dom.hi, NVAR);
  fr.cfp.alloc(gc.dom.lo, gc.dom.hi, NVAR);
  return fr;
}

// Coarse data at time t from the old/new coarse states (StateData::getData
// then FillPatchSingleLevel's time interpolation).
struct CoarseAt {
  const Fab* old_s;
  const Fab* new_s;
  double t0, t1, t;
  int mode;  // 0 new, 1 old, 2 interpolate
  double alpha, beta;
  // StateData::getData: the new (old) data when t is within
  // 1e-3 (t1 - t0) of t1 (t0), else both, combined by LinComb with
  // alpha = (t1 - t)/(t1 - t0), beta = (t - t0)/(t1 - t0).
  void init() {
    const double teps = (t1 - t0) * 1.e-3;
    if (t > t1 - teps && t < t1 + teps) mode = 0;
    else if (t > t0 - teps && t < t0 + teps) mode = 1;
    else {
      mode = 2;
      alpha = (t1 - t) / (t1 - t0);
      beta = (t - t0) / (t1 - t0);
    }
  }
  double operator()(int i, int j, int k, int n) const {
    if (mode == 0) return (*new_s)(i, j, k, n);
    if (mode == 1) return (*old_s)(i, j, k, n);
    return alpha * (*old_s)(i, j, k, n) + beta * (*new_s)(i, j, k, n);
  }
};

// Conservative linear interpolation of component n to fine cell (fi,fj,fk)
// (AMReX CellConservativeLinear with limiting, ratio 2).  Per direction an
// MC-limited slope: dc = (u+ - u-)/2, s = min(|2(u+ - u)|, |2(u - u-)|) when
// those agree in sign (else 0), s = sign(dc) min(s, |dc|); then one factor
// alpha <= 1 for all three slopes keeps every fine child inside the min/max
// of the 27 coarse neighbours (the children lie at most (r-1)/(2r) = 1/4 of
// a slope from the centre).  fine = u + ox*sx + oy*sy + oz*sz, o = -+1/4.
double cons_interp(const CoarseAt& C, const Grid& gc, int fi, int fj, int fk, int n) {
  const int f[3] = {fi, fj, fk};
  int c[3];
  for (int d = 0; d < 3; ++d) c[d] = (f[d] >= 0) ? f[d] / RR : -((-f[d] + RR - 1) / RR);
  auto at = [&](int di, int dj, int dk) {
    return C(wrap(c[0] + di, gc.dom.lo[0], gc.n[0]), wrap(c[1] + dj, gc.dom.lo[1], gc.n[1]),
             wrap(c[2] + dk, gc.dom.lo[2], gc.n[2]), n);
  };
  const double uc = at(0, 0, 0);
  double sl[3];
  const int e[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int d = 0; d < 3; ++d) {
    const double up = at(e[d][0], e[d][1], e[d][2]);
    const double um = at(-e[d][0], -e[d][1], -e[d][2]);
    const double dc = 0.5 * (up - um);
    const double df = 2.0 * (up - uc);
    const double db = 2.0 * (uc - um);
    double sv = (df * db >= 0.0) ? std::min(std::fabs(df), std::fabs(db)) : 0.0;
    sv = std::copysign(1.0, dc) * std::min(sv, std::fabs(dc));
    sl[d] = sv;
  }
  double alpha = 1.0;
  if (sl[0] != 0.0 || sl[1] != 0.0 || sl[2] != 0.0) {
    const double dumax = std::fabs(sl[0]) * 0.25 + std::fabs(sl[1]) * 0.25 + std::fabs(sl[2]) * 0.25;
    double umax = uc, umin = uc;
    for (int dk = -1; dk <= 1; ++dk)
      for (int dj = -1; dj <= 1; ++dj)
        for (int di = -1; di <= 1; ++di) {
          const double v = at(di, dj, dk);
          umax = std::max(umax, v);
          umin = std::min(umin, v);
        }
    if (dumax * alpha > (umax - uc)) alpha = (umax - uc) / dumax;
    if (dumax * alpha > (uc - umin)) alpha = (uc - umin) / dumax;
  }
  double off[3];
  for (int d = 0; d < 3; ++d) off[d] = (f[d] - RR * c[d] == 0) ? -0.25 : 0.25;
  return uc + off[0] * (sl[0] * alpha) + off[1] * (sl[1] * alpha) + off[2] * (sl[2] * alpha);
}

// FillBoundary of the fine level: every ghost cell of grow(box, 4) that a
// fine box covers (through the periodic domain) gets that box's valid value.
void fine_fill_boundary(const Fine& fn, const FluxReg& fr, std::vector<Fab>& Bv) {
  int fdlo[3], fn_n[3];
  for (int d = 0; d < 3; ++d) {
    fdlo[d] = fn.L.dom_lo[d];
    fn_n[d] = fn.L.dom_hi[d] - fn.L.dom_lo[d] + 1;
  }
  const int nb = int(fn.boxes.size());
  for (int b = 0; b < nb; ++b) {
    const Box3& bx = fn.boxes[b];
    for_box(grow(bx, 4), [&](int i, int j, int k) {
      const bool valid = i >= bx.lo[0] && i <= bx.hi[0] && j >= bx.lo[1] && j <= bx.hi[1] &&
                         k >= bx.lo[2] && k <= bx.hi[2];
      if (valid) return;
      const int wi = wrap(i, fdlo[0], fn_n[0]), wj = wrap(j, fdlo[1], fn_n[1]),
                wk = wrap(k, fdlo[2], fn_n[2]);
      const int ob = fr.box_at(wi / RR, wj / RR, wk / RR);
      if (ob >= 0)
        for (int n = 0; n < NVAR; ++n) Bv[b](i, j, k, n) = Bv[ob](wi, wj, wk, n);
    });
  }
}

// FillPatchTwoLevels + clean_state of every fine box's Sborder from the fine
// valid data src and the coarse data at time t.
void fine_expand(const Eos& eos, const orc_params& p, Fine& fn, const Grid& gc,
                 const FluxReg& fr, const std::vector<Fab>& src, const CoarseAt& C,
                 std::vector<Fab>& Bv) {
  const int nb = int(fn.boxes.size());
  const int nth = nthreads_of(fn.L);
  int fdlo[3], fn_n[3];
  for (int d = 0; d < 3; ++d) {
    fdlo[d] = fn.L.dom_lo[d];
    fn_n[d] = fn.L.dom_hi[d] - fn.L.dom_lo[d] + 1;
  }
  // valid cells, then enforce_min_density and normalize_species on them
#pragma omp parallel for num_threads(nth) schedule(dynamic)
  for (int b = 0; b < nb; ++b) {
    const Box3& bx = fn.boxes[b];
    for_box(bx, [&](int i, int j, int k) {
      for (int n = 0; n < NVAR; ++n) Bv[b](i, j, k, n) = src[b](i, j, k, n);
    });
    enforce_min_density_tile(eos, p, Bv[b], bx);
    for_box(bx, [&](int i, int j, int k) { normalize_species_cell(Bv[b], i, j, k); });
  }
  // ghost cells: fine-fine from the other boxes' cleaned valid data
  // (FillBoundary at the end of normalize_species), coarse-fine from the
  // interpolated coarse data; then computeTemp on every cell
  fine_fill_boundary(fn, fr, Bv);
#pragma omp parallel for num_threads(nth) schedule(dynamic)
  for (int b = 0; b < nb; ++b) {
    const Box3& bx = fn.boxes[b];
    for_box(grow(bx, 4), [&](int i, int j, int k) {
      const bool valid = i >= bx.lo[0] && i <= bx.hi[0] && j >= bx.lo[1] && j <= bx.hi[1] &&
                         k >= bx.lo[2] && k <= bx.hi[2];
      if (valid) return;
      const int wi = wrap(i, fdlo[0], fn_n[0]), wj = wrap(j, fdlo[1], fn_n[1]),
                wk = wrap(k, fdlo[2], fn_n[2]);
      if (fr.box_at(wi / RR, wj / RR, wk / RR) < 0)
        for (int n = 0; n < NVAR; ++n) Bv[b](i, j, k, n) = cons_interp(C, gc, i, j, k, n);
    });
  }
#pragma omp parallel for num_threads(nth) schedule(dynamic)
  for (int b = 0; b < nb; ++b) {
    for_box(grow(fn.boxes[b], 4), [&](int i, int j, int k) { compute_temp_cell(eos, p, Bv[b], i, j, k); });
  }
}

// YAFluxRegister::FineAdd for one fine hydro call, box after box: for
// each side of each fine box, every coarse cell just outside it that no
// fine box covers gets the fine fluxes of its 4 fine faces (slower
// transverse index outer), scaled by dt_f/(vol_f * ratio^3); subtracted on
// the box's low side, added on its high side.  The sums go to cfp, which
// the reflux adds to the CrseAdd sums.
void fine_add(FluxReg& fr, const Grid& gc, const Fine& fn, double dtdx) {
  for (size_t b = 0; b < fn.boxes.size(); ++b) {
    Box3 cb;
    for (int d = 0; d < 3; ++d) {
      cb.lo[d] = fn.boxes[b].lo[d] / RR;
      cb.hi[d] = fn.boxes[b].hi[d] / RR;
    }
    for (int d = 0; d < 3; ++d) {
      const int t1 = (d == 0) ? 1 : 0;  // faster transverse index
      const int t2 = (d == 2) ? 1 : 2;  // slower transverse index
      for (int side = 0; side < 2; ++side) {
        Box3 adj = cb;
        adj.lo[d] = adj.hi[d] = side ? cb.hi[d] + 1 : cb.lo[d] - 1;
        const int fface = side ? RR * (cb.hi[d] + 1) : RR * cb.lo[d];
        for (int n = 0; n < NVAR; ++n)
          for_box(adj, [&](int i, int j, int k) {
            if (fr.box_at(i, j, k) >= 0) return;
            const int cc[3] = {i, j, k};
            int w[3];
            for (int e = 0; e < 3; ++e) w[e] = wrap(cc[e], gc.dom.lo[e], gc.n[e]);
            double& acc = fr.cfp(w[0], w[1], w[2], n);
            for (int a2 = 0; a2 < RR; ++a2)
              for (int a1 = 0; a1 < RR; ++a1) {
                int fi[3];
                fi[d] = fface;
                fi[t1] = RR * cc[t1] + a1;
                fi[t2] = RR * cc[t2] + a2;
                const double v = dtdx * fn.F[d][b](fi[0], fi[1], fi[2], n);
                if (side) acc += v;
                else acc -= v;
              }
          });
      }
    }
  }
}

double est_dt_boxes(const Eos& eos, const orc_params& p, const orc_level& L,
                    const std::vector<Box3>& boxes, const std::vector<Fab>& S) {
  if (p.fixed_dt > 0.0) return p.fixed_dt;
  double estdt = p.max_dt;
  double estdt_hydro = p.max_dt / p.cfl;
  double dt = std::numeric_limits<double>::max();
  for (size_t b = 0; b < boxes.size(); ++b) {
    for_box(boxes[b], [&](int i, int j, int k) {
      const Fab& U = S[b];
      const double rho = U(i, j, k, URHO);
      const double rhoInv = 1.0 / rho;
      const double eint = U(i, j, k, UEINT) / rho;
      const double pres = eos.rey2p(rho, eint);
      const double c = std::sqrt(eos.gamma * pres / rho);
      dt = std::min(dt, L.dx[0] / (c + std::fabs(U(i, j, k, UMX) * rhoInv)));
      dt = std::min(dt, L.dx[1] / (c + std::fabs(U(i, j, k, UMY) * rhoInv)));
      dt = std::min(dt, L.dx[2] / (c + std::fabs(U(i, j, k, UMZ) * rhoInv)));
    });
  }
  estdt_hydro = std::min(estdt_hydro, dt);
  estdt_hydro *= p.cfl;
  if (estdt_hydro < estdt) estdt = estdt_hydro;
  return estdt;
}

long clean_boxes(const Eos& eos, const orc_params& p, Fine& fn, std::vector<Fab>& S) {
  long nerr = 0;
  const int nb = int(fn.boxes.size());
  const int nth = nthreads_of(fn.L);
#pragma omp parallel for num_threads(nth) reduction(+ : nerr) schedule(dynamic)
  for (int b = 0; b < nb; ++b) {
    nerr += enforce_min_density_tile(eos, p, S[b], fn.boxes[b]);
    for_box(fn.boxes[b], [&](int i, int j, int k) { normalize_species_cell(S[b], i, j, k); });
    for_box(fn.boxes[b], [&](int i, int j, int k) { compute_temp_cell(eos, p, S[b], i, j, k); });
  }
  return nerr;
}

// hydro of every fine box (construct_hydro_source on level 1), then FineAdd.
long fine_hydro(const orc_params& p, Fine& fn, std::vector<Fab>& Bv, std::vector<Fab>& dsdt,
                const std::vector<Fab>* src, double dt, FluxReg& fr, const Grid& gc,
                double dtdx_fine) {
  long nerr = 0;
  const int nb = int(fn.boxes.size());
  const int nth = nthreads_of(fn.L);
#pragma omp parallel for num_threads(nth) reduction(+ : nerr) schedule(dynamic)
  for (int b = 0; b < nb; ++b) {
    const Box3& bx = fn.boxes[b];
    for_box(bx, [&](int i, int j, int k) {
      for (int n = 0; n < NVAR; ++n) dsdt[b](i, j, k, n) = 0.0;
    });
    nerr += orc_hydro_box(&p, bx.lo, bx.hi, fn.L.dom_lo, fn.L.dom_hi, fn.L.bc_lo, fn.L.bc_hi,
                          Bv[b].p, Bv[b].lo, Bv[b].hi, src ? (*src)[b].p : nullptr, dsdt[b].p, dsdt[b].lo,
                          dsdt[b].hi, fn.F[0][b].p, fn.F[1][b].p, fn.F[2][b].p, fn.L.dx, dt);
  }
  fine_add(fr, gc, fn, dtdx_fine);
  return nerr;
}

// One fine-level CAMR::advance + post_timestep (finest level).
long fine_advance(const Eos& eos, const orc_params& p, Fine& fn, const Grid& gc, FluxReg& fr,
                  const Fab& c_old, const Fab& c_new, double tc0, double tc1, double tf_old,
                  double tf_new, double dt) {
  long nerr = 0;
  const int nb = int(fn.boxes.size());
  const double volf = fn.L.dx[0] * fn.L.dx[1] * fn.L.dx[2];
  const double dtdx_f = ((p.do_mol ? 0.5 : 1.0) * dt) / (volf * double(RR * RR * RR));
  for (int b = 0; b < nb; ++b) {
    for_box(fn.boxes[b], [&](int i, int j, int k) {
      for (int n = 0; n < NVAR; ++n) fn.S_old[b](i, j, k, n) = fn.S[b](i, j, k, n);
    });
  }
  nerr += clean_boxes(eos, p, fn, fn.S_old);
  CoarseAt C0{&c_old, &c_new, tc0, tc1, tf_old, 0, 0.0, 0.0};
  C0.init();
  fine_expand(eos, p, fn, gc, fr, fn.S_old, C0, fn.B);
  for (int b = 0; b < nb; ++b) {
    for_box(fn.boxes[b], [&](int i, int j, int k) {
      for (int n = 0; n < NVAR; ++n) fn.S[b](i, j, k, n) = fn.B[b](i, j, k, n);
      if (p.add_grav_src) {
        double src[NVAR];
        for (int n = 0; n < NVAR; ++n) src[n] = 0.0;
        src[UMZ] = p.const_grav * fn.S_old[b](i, j, k, URHO);
        src[UEDEN] = p.const_grav * fn.S_old[b](i, j, k, UMZ);
        for (int n = 0; n < NVAR; ++n) fn.S[b](i, j, k, n) += dt * src[n];
      }
    });
  }
  if (p.do_mol) {
    nerr += fine_hydro(p, fn, fn.B, fn.dsdt, nullptr, dt, fr, gc, dtdx_f);
    for (int b = 0; b < nb; ++b)
      for_box(fn.boxes[b], [&](int i, int j, int k) {
        for (int n = 0; n < NVAR; ++n) fn.S[b](i, j, k, n) += dt * fn.dsdt[b](i, j, k, n);
      });
    CoarseAt C1{&c_old, &c_new, tc0, tc1, tf_new, 0, 0.0, 0.0};
    C1.init();
    fine_expand(eos, p, fn, gc, fr, fn.S, C1, fn.B2);
    nerr += fine_hydro(p, fn, fn.B2, fn.dsdt2, nullptr, dt, fr, gc, dtdx_f);
    for (int b = 0; b < nb; ++b)
      for_box(fn.boxes[b], [&](int i, int j, int k) {
        for (int n = 0; n < NVAR; ++n)
          fn.S[b](i, j, k, n) = 0.5 * fn.B2[b](i, j, k, n) + 0.5 * fn.S_old[b](i, j, k, n);
        for (int n = 0; n < NVAR; ++n) fn.S[b](i, j, k, n) += 0.5 * dt * fn.dsdt2[b](i, j, k, n);
      });
  } else {
    // sources_for_hydro: 0 + 1.0 * old source on valid cells, FillBoundary
    // from the other fine boxes, zero on the coarse-fine ghost cells.
    for (int b = 0; b < nb; ++b) {
      for (auto& v : fn.sfh[b].own) v = 0.0;
      if (p.add_grav_src)
        for_box(fn.boxes[b], [&](int i, int j, int k) {
          double src[NVAR];
          for (int n = 0; n < NVAR; ++n) src[n] = 0.0;
          src[UMZ] = p.const_grav * fn.S_old[b](i, j, k, URHO);
          src[UEDEN] = p.const_grav * fn.S_old[b](i, j, k, UMZ);
          for (int n = 0; n < NVAR; ++n) fn.sfh[b](i, j, k, n) += 1.0 * src[n];
        });
    }
    if (p.add_grav_src) fine_fill_boundary(fn, fr, fn.sfh);
    nerr += fine_hydro(p, fn, fn.B, fn.dsdt, &fn.sfh, dt, fr, gc, dtdx_f);
    for (int b = 0; b < nb; ++b)
      for_box(fn.boxes[b], [&](int i, int j, int k) {
        for (int n = 0; n < NVAR; ++n) fn.S[b](i, j, k, n) += dt * fn.dsdt[b](i, j, k, n);
      });
  }
  nerr += clean_boxes(eos, p, fn, fn.S);
  if (p.add_grav_src) {
    for (int b = 0; b < nb; ++b)
      for_box(fn.boxes[b], [&](int i, int j, int k) {
        double src[NVAR];
        for (int n = 0; n < NVAR; ++n) src[n] = 0.0;
        src[UMZ] = 0.5 * p.const_grav * (fn.S[b](i, j, k, URHO) - fn.S_old[b](i, j, k, URHO));
        src[UEDEN] = 0.5 * p.const_grav * (fn.S[b](i, j, k, UMZ) - fn.S_old[b](i, j, k, UMZ));
        for (int n = 0; n < NVAR; ++n) fn.S[b](i, j, k, n) += dt * src[n];
      });
    nerr += clean_boxes(eos, p, fn, fn.S);
  }
  nerr += clean_boxes(eos, p, fn, fn.S);  // post_timestep of the finest level
  return nerr;
}

void avg_down(const Grid& gc, const Fine& fn, const Fab& Sc) {
  for (size_t b = 0; b < fn.boxes.size(); ++b) {
    Box3 cb;
    for (int d = 0; d < 3; ++d) {
      cb.lo[d] = fn.boxes[b].lo[d] / RR;
      cb.hi[d] = fn.boxes[b].hi[d] / RR;
    }
    const double volfrac = 1.0 / static_cast<double>(RR * RR * RR);
    for_box(cb, [&](int i, int j, int k) {
      for (int n = 0; n < NVAR; ++n) {
        double c = 0.0;
        for (int kr = 0; kr < RR; ++kr)
          for (int jr = 0; jr < RR; ++jr)
            for (int ir = 0; ir < RR; ++ir)
              c += fn.S[b](RR * i + ir, RR * j + jr, RR * k + kr, n);
        Sc(i, j, k, n) = volfrac * c;
      }
    });
  }
  (void)gc;
}

}  // namespace
}  // namespace orc

extern "C" long orc_amr_run(const orc_params* p, const orc_level* lev0, int nbox,
                            const int* boxes, double* S0, double* S1, int nsteps, int do_init,
                            int first_step, double* clock, double* dt_hist) {
  using namespace orc;
  const Eos eos{p->eos_gamma};
  const orc_level& Lc = *lev0;
  const Grid gc = make_grid(Lc);
  Fab Sc;
  Sc.view(S0, gc.dom.lo, gc.dom.hi, NVAR);
  Fine fn;
  fn.L = Lc;
  for (int d = 0; d < 3; ++d) {
    fn.L.dom_lo[d] = Lc.dom_lo[d] * RR;
    fn.L.dom_hi[d] = (Lc.dom_hi[d] + 1) * RR - 1;
    fn.L.dx[d] = Lc.dx[d] / RR;
    fn.L.max_grid_size[d] = 0;
    fn.L.tile_size[d] = 0;
  }
  size_t off = 0;
  for (int b = 0; b < nbox; ++b) {
    Box3 bx;
    for (int d = 0; d < 3; ++d) {
      bx.lo[d] = boxes[6 * b + d];
      bx.hi[d] = boxes[6 * b + 3 + d];
    }
    fn.boxes.push_back(bx);
  }
  const int nb = nbox;
  fn.S.resize(nb);
  fn.S_old.resize(nb);
  fn.B.resize(nb);
  fn.B2.resize(nb);
  fn.dsdt.resize(nb);
  fn.dsdt2.resize(nb);
  fn.sfh.resize(nb);
  for (int d = 0; d < 3; ++d) {
    fn.fbuf[d].resize(nb);
    fn.F[d].resize(nb);
  }
  for (int b = 0; b < nb; ++b) {
    const Box3& bx = fn.boxes[b];
    fn.S[b].view(S1 + off, bx.lo, bx.hi, NVAR);
    off += size_t(fn.S[b].sn) * NVAR;
    fn.S_old[b].alloc(bx.lo, bx.hi, NVAR);
    const Box3 g4 = grow(bx, 4);
    fn.B[b].alloc(g4.lo, g4.hi, NVAR);
    fn.B2[b].alloc(g4.lo, g4.hi, NVAR);
    fn.sfh[b].alloc(g4.lo, g4.hi, NVAR);
    fn.dsdt[b].alloc(bx.lo, bx.hi, NVAR);
    fn.dsdt2[b].alloc(bx.lo, bx.hi, NVAR);
    for (int d = 0; d < 3; ++d) {
      const Box3 fb = faces(bx, d);
      fn.fbuf[d][b].resize(size_t(fb.hi[0] - fb.lo[0] + 1) * (fb.hi[1] - fb.lo[1] + 1) *
                           (fb.hi[2] - fb.lo[2] + 1) * NVAR);
      fn.F[d][b].view(fn.fbuf[d][b].data(), fb.lo, fb.hi, NVAR);
    }
  }
  FluxReg fr = make_fluxreg(gc, Lc, fn.boxes);
  Work w;
  alloc_work(gc, w);
  long nerr = 0;
  if (do_init) {
    // CAMR::initData epilogue on both levels, then post_init's avgDown.
    orc_init_finalize(p, &Lc, S0);
    for (int b = 0; b < nb; ++b) {
      for_box(fn.boxes[b], [&](int i, int j, int k) {
        Fab& U = fn.S[b];
        const double rhoInv = 1.0 / U(i, j, k, URHO);
        const double u = U(i, j, k, UMX) * rhoInv;
        const double v = U(i, j, k, UMY) * rhoInv;
        const double ww = U(i, j, k, UMZ) * rhoInv;
        U(i, j, k, UEDEN) = U(i, j, k, UEINT) + 0.5 * U(i, j, k, URHO) * (u * u + v * v + ww * ww);
        compute_temp_cell(eos, *p, U, i, j, k);
      });
    }
    avg_down(gc, fn, Sc);
  }
  double dtl[2] = {clock[2], clock[3]};
  double tc_new = clock[0], tf_new = clock[1];
  const int ncyc[2] = {1, RR};
  for (int step = 0; step < nsteps; ++step) {
    // Amr::computeInitialDt / CAMR::computeNewDt over both levels
    double dtm[2];
    dtm[0] = est_dt(eos, *p, Lc, gc, Sc);
    dtm[1] = est_dt_boxes(eos, *p, fn.L, fn.boxes, fn.S);
    if (step == 0 && first_step) {
      for (int l = 0; l < 2; ++l)
        dtm[l] = (p->initial_dt > 0.0) ? p->initial_dt : p->init_shrink * dtm[l];
    } else if (p->fixed_dt <= 0.0) {
      for (int l = 0; l < 2; ++l) dtm[l] = std::min(dtm[l], p->change_max * dtl[l]);
    }
    double dt_0 = std::numeric_limits<double>::max();
    int nf = 1;
    for (int l = 0; l < 2; ++l) {
      nf *= ncyc[l];
      dt_0 = std::min(dt_0, nf * dtm[l]);
    }
    nf = 1;
    for (int l = 0; l < 2; ++l) {
      nf *= ncyc[l];
      dtl[l] = dt_0 / nf;
    }
    if (dt_hist) {
      dt_hist[2 * step] = dtl[0];
      dt_hist[2 * step + 1] = dtl[1];
    }
    // level 0: flux register reset, advance (CrseAdd), keep old/new
    for (auto& v : fr.d.own) v = 0.0;
    for (auto& v : fr.cfp.own) v = 0.0;
    const double tc_old = tc_new;
    tc_new = tc_new + dtl[0];
    nerr += advance_one(eos, *p, Lc, gc, Sc, w, dtl[0], &fr, false);
    // level 1: two subcycled steps
    Fab c_new_copy(gc.dom.lo, gc.dom.hi, NVAR);
    std::memcpy(c_new_copy.p, Sc.p, sizeof(double) * size_t(gc.ncell) * NVAR);
    for (int sc = 0; sc < RR; ++sc) {
      const double tf_old = tf_new;
      tf_new = tf_new + dtl[1];
      nerr += fine_advance(eos, *p, fn, gc, fr, w.S_old, c_new_copy, tc_old, tc_new, tf_old,
                           tf_new, dtl[1]);
    }
    // post_timestep(0): reflux, avgDown, clean_state
    for_box(gc.dom, [&](int i, int j, int k) {
      for (int n = 0; n < NVAR; ++n) {
        const double dcorr = fr.d(i, j, k, n) + fr.cfp(i, j, k, n);
        Sc(i, j, k, n) = Sc(i, j, k, n) + dcorr;
      }
    });
    avg_down(gc, fn, Sc);
    nerr += clean_state_valid(eos, *p, Lc, gc, Sc);
  }
  clock[0] = tc_new;
  clock[1] = tf_new;
  clock[2] = dtl[0];
  clock[3] = dtl[1];
  return nerr;
}

// The two-level flux register alone, on fluxes the caller supplies: CrseAdd
// of each coarse box's face fluxes for each of ncrse coarse hydro calls
// (scale dtdx_c), then FineAdd of every
// fine box's face fluxes for each of ncall fine hydro calls (scale dtdx_f),
// then the reflux of post_timestep, S0 += d + cfp over the whole coarse
// domain -- the same make_fluxreg / crse_add / fine_add and reflux loop as
// orc_amr_run.  The domain must be periodic (as orc_amr_run's).
// cflux: for each coarse call, each coarse box c, d = 0..2, NVAR comps on
// faces(box c, d);
// fflux: for each call, each fine box b, d = 0..2, NVAR comps on
// faces(fine box b, d); every fab with i fastest and the component slowest.
extern "C" void orc_fluxreg_reflux(const orc_level* lev0, int ncbox, const int* cboxes,
                                   int ncrse, const double* cflux, double dtdx_c, int nfbox,
                                   const int* fboxes, int ncall, const double* fflux,
                                   double dtdx_f, double* S0) {
  using namespace orc;
  const orc_level& Lc = *lev0;
  const Grid gc = make_grid(Lc);
  Fab Sc;
  Sc.view(S0, gc.dom.lo, gc.dom.hi, NVAR);
  Fine fn;
  for (int b = 0; b < nfbox; ++b) {
    Box3 bx;
    for (int d = 0; d < 3; ++d) {
      bx.lo[d] = fboxes[6 * b + d];
      bx.hi[d] = fboxes[6 * b + 3 + d];
    }
    fn.boxes.push_back(bx);
  }
  FluxReg fr = make_fluxreg(gc, Lc, fn.boxes);
  for (auto& v : fr.d.own) v = 0.0;
  for (auto& v : fr.cfp.own) v = 0.0;
  size_t off = 0;
  for (int call = 0; call < ncrse; ++call)
    for (int c = 0; c < ncbox; ++c) {
      Box3 bx;
      for (int d = 0; d < 3; ++d) {
        bx.lo[d] = cboxes[6 * c + d];
        bx.hi[d] = cboxes[6 * c + 3 + d];
      }
      Fab f[3];
      for (int d = 0; d < 3; ++d) {
        const Box3 fb = faces(bx, d);
        f[d].view(const_cast<double*>(cflux) + off, fb.lo, fb.hi, NVAR);
        off += size_t(f[d].sn) * NVAR;
      }
      crse_add(fr, bx, f, dtdx_c);
    }
  for (int d = 0; d < 3; ++d) fn.F[d].resize(nfbox);
  off = 0;
  for (int call = 0; call < ncall; ++call) {
    for (int b = 0; b < nfbox; ++b)
      for (int d = 0; d < 3; ++d) {
        const Box3 fb = faces(fn.boxes[b], d);
        fn.F[d][b].view(const_cast<double*>(fflux) + off, fb.lo, fb.hi, NVAR);
        off += size_t(fn.F[d][b].sn) * NVAR;
      }
    fine_add(fr, gc, fn, dtdx_f);
  }
  for_box(gc.dom, [&](int i, int j, int k) {
    for (int n = 0; n < NVAR; ++n) {
      const double dcorr = fr.d(i, j, k, n) + fr.cfp(i, j, k, n);
      Sc(i, j, k, n) = Sc(i, j, k, n) + dcorr;
    }
  });
}

// avgDown alone (the avg_down of orc_amr_run's post_timestep): S1 holds the
// fine boxes' valid states back to back (NVAR comps each, i fastest); the
// coarse cells they cover in S0 become the averages of their children.
extern "C" void orc_avg_down(const orc_level* lev0, int nfbox, const int* fboxes, double* S1,
                             double* S0) {
  using namespace orc;
  const Grid gc = make_grid(*lev0);
  Fab Sc;
  Sc.view(S0, gc.dom.lo, gc.dom.hi, NVAR);
  Fine fn;
  fn.S.resize(nfbox);
  size_t off = 0;
  for (int b = 0; b < nfbox; ++b) {
    Box3 bx;
    for (int d = 0; d < 3; ++d) {
      bx.lo[d] = fboxes[6 * b + d];
      bx.hi[d] = fboxes[6 * b + 3 + d];
    }
    fn.boxes.push_back(bx);
    fn.S[b].view(S1 + off, bx.lo, bx.hi, NVAR);
    off += size_t(fn.S[b].sn) * NVAR;
  }
  avg_down(gc, fn, Sc);
}

// The ghost cells of FillPatchTwoLevels alone (fine_expand's fill, without
// its cleaning passes): Bv holds each fine box grown by 4 back to back (NVAR
// comps each, i fastest) with the valid cells set; every ghost cell that a
// fine box covers (through the periodic domain) gets that box's valid
// value, every other one the conservative interpolation of the coarse data
// at time t from c_old (time t0) and c_new (time t1).
extern "C" void orc_fine_fill_ghosts(const orc_level* lev0, int nfbox, const int* fboxes,
                                     double* Bv, const double* c_old, const double* c_new,
                                     double t0, double t1, double t) {
  using namespace orc;
  const orc_level& Lc = *lev0;
  const Grid gc = make_grid(Lc);
  Fab Co, Cn;
  Co.view(const_cast<double*>(c_old), gc.dom.lo, gc.dom.hi, NVAR);
  Cn.view(const_cast<double*>(c_new), gc.dom.lo, gc.dom.hi, NVAR);
  Fine fn;
  fn.L = Lc;
  for (int d = 0; d < 3; ++d) {
    fn.L.dom_lo[d] = Lc.dom_lo[d] * RR;
    fn.L.dom_hi[d] = (Lc.dom_hi[d] + 1) * RR - 1;
    fn.L.dx[d] = Lc.dx[d] / RR;
  }
  std::vector<Fab> B(nfbox);
  size_t off = 0;
  for (int b = 0; b < nfbox; ++b) {
    Box3 bx;
    for (int d = 0; d < 3; ++d) {
      bx.lo[d] = fboxes[6 * b + d];
      bx.hi[d] = fboxes[6 * b + 3 + d];
    }
    fn.boxes.push_back(bx);
    const Box3 g4 = grow(bx, 4);
    B[b].view(Bv + off, g4.lo, g4.hi, NVAR);
    off += size_t(B[b].sn) * NVAR;
  }
  const FluxReg fr = make_fluxreg(gc, Lc, fn.boxes);
  CoarseAt C{&Co, &Cn, t0, t1, t, 0, 0.0, 0.0};
  C.init();
  fine_fill_boundary(fn, fr, B);
  int fdlo[3], fn_n[3];
  for (int d = 0; d < 3; ++d) {
    fdlo[d] = fn.L.dom_lo[d];
    fn_n[d] = fn.L.dom_hi[d] - fn.L.dom_lo[d] + 1;
  }
  for (int b = 0; b < nfbox; ++b) {
    const Box3& bx = fn.boxes[b];
    for_box(grow(bx, 4), [&](int i, int j, int k) {
      const bool valid = i >= bx.lo[0] && i <= bx.hi[0] && j >= bx.lo[1] && j <= bx.hi[1] &&
                         k >= bx.lo[2] && k <= bx.hi[2];
      if (valid) return;
      const int wi = wrap(i, fdlo[0], fn_n[0]), wj = wrap(j, fdlo[1], fn_n[1]),
                wk = wrap(k, fdlo[2], fn_n[2]);
      if (fr.box_at(wi / RR, wj / RR, wk / RR) < 0)
        for (int n = 0; n < NVAR; ++n) B[b](i, j, k, n) = cons_interp(C, gc, i, j, k, n);
    });
  }
}

namespace orc {
namespace {
}  // namespace
}  // namespace orc

using namespace orc;

extern "C" void orc_default_params(orc_params* p) { default_params(p); }

extern "C" void orc_init_finalize(const orc_params* p, const orc_level* lev, double* state) {
  const Grid g = make_grid(*lev);
  const Eos eos{p->eos_gamma};
  Fab S;
  S.view(state, g.dom.lo, g.dom.hi, NVAR);
  const int nth = nthreads_of(*lev);
  // enforce_consistent_e (Source/CAMR.cpp:910-939)
  par_cells(g, nth, [&](int i, int j, int k) {
    const double rhoInv = 1.0 / S(i, j, k, URHO);
    const double u = S(i, j, k, UMX) * rhoInv;
    const double v = S(i, j, k, UMY) * rhoInv;
    const double w = S(i, j, k, UMZ) * rhoInv;
    S(i, j, k, UEDEN) = S(i, j, k, UEINT) + 0.5 * S(i, j, k, URHO) * (u * u + v * v + w * w);
  });
  par_cells(g, nth, [&](int i, int j, int k) { compute_temp_cell(eos, *p, S, i, j, k); });
}

extern "C" double orc_est_dt(const orc_params* p, const orc_level* lev, const double* state) {
  const Grid g = make_grid(*lev);
  const Eos eos{p->eos_gamma};
  Fab S;
  S.view(const_cast<double*>(state), g.dom.lo, g.dom.hi, NVAR);
  return est_dt(eos, *p, *lev, g, S);
}

extern "C" long orc_advance(const orc_params* p, const orc_level* lev, double* state, int nsteps,
                            int first_step, double* dt_prev, double* dt_hist) {
  const Grid g = make_grid(*lev);
  const Eos eos{p->eos_gamma};
  Fab S;
  S.view(state, g.dom.lo, g.dom.hi, NVAR);
  Work w;
  alloc_work(g, w);
  long nerr = 0;
  double dt_level = *dt_prev;
  for (int s = 0; s < nsteps; ++s) {
    double dt;
    if (first_step && s == 0) {
      // computeInitialDt (Source/CAMR.cpp:638-676) / initialTimeStep (:473-487)
      double init_dt;
      if (p->initial_dt > 0.0) init_dt = p->initial_dt;
      else init_dt = p->init_shrink * est_dt(eos, *p, *lev, g, S);
      double dt_0 = std::numeric_limits<double>::max();
      dt_0 = std::min(dt_0, 1 * init_dt);
      dt = dt_0 / 1;
    } else {
      // computeNewDt (Source/CAMR.cpp:566-635), single level, no regrid
      double dt_min = est_dt(eos, *p, *lev, g, S);
      if (p->fixed_dt <= 0.0) dt_min = std::min(dt_min, p->change_max * dt_level);
      double dt_0 = std::numeric_limits<double>::max();
      dt_0 = std::min(dt_0, 1 * dt_min);
      dt = dt_0 / 1;
    }
    nerr += advance_one(eos, *p, *lev, g, S, w, dt);
    dt_level = dt;
    if (dt_hist) dt_hist[s] = dt;
  }
  *dt_prev = dt_level;
  return nerr;
}

extern "C" long orc_advance_fixed_dt(const orc_params* p, const orc_level* lev, double* state,
                                     int nsteps, const double* dts) {
  const Grid g = make_grid(*lev);
  const Eos eos{p->eos_gamma};
  Fab S;
  S.view(state, g.dom.lo, g.dom.hi, NVAR);
  Work w;
  alloc_work(g, w);
  long nerr = 0;
  for (int s = 0; s < nsteps; ++s) nerr += advance_one(eos, *p, *lev, g, S, w, dts[s]);
  return nerr;
}

extern "C" void orc_expand_state(const orc_params* p, const orc_level* lev, const double* state,
                                 int ng, double* border) {
  const Grid g = make_grid(*lev);
  const Eos eos{p->eos_gamma};
  Fab S, B;
  S.view(const_cast<double*>(state), g.dom.lo, g.dom.hi, NVAR);
  const Box3 bg = grow(g.dom, ng);
  B.view(border, bg.lo, bg.hi, NVAR);
  expand_state(eos, *p, *lev, g, S, B);
}

extern "C" void orc_clean_state(const orc_params* p, const orc_level* lev, double* state) {
  const Grid g = make_grid(*lev);
  const Eos eos{p->eos_gamma};
  Fab S;
  S.view(state, g.dom.lo, g.dom.hi, NVAR);
  clean_state_valid(eos, *p, *lev, g, S);
}
