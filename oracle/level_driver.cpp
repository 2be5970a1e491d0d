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
long hydro_level(const orc_params& p, const orc_level& L, const Grid& g, const Fab& B,
                 const Fab* src, const Fab& dsdt, double dt) {
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
                 const Fab& S, Work& w, double dt) {
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
    nerr += hydro_level(p, L, g, w.B, nullptr, w.dsdt, dt);
    par_cells(g, nth, [&](int i, int j, int k) {
      for (int n = 0; n < NVAR; ++n) S(i, j, k, n) += dt * w.dsdt(i, j, k, n);
    });
    nerr += expand_state(eos, p, L, g, S, w.B2);
    nerr += hydro_level(p, L, g, w.B2, nullptr, w.dsdt2, dt);
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
    nerr += hydro_level(p, L, g, w.B, &w.sfh, w.dsdt, dt);
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
  nerr += clean_state_valid(eos, p, L, g, S);
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
