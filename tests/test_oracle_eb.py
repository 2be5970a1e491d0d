"""CPU tests of the EB oracle (the reference's EB hydro kernels built with
AMREX_USE_EB against the AMReX stand-in, oracle/_ref/libcamr_ref_eb.so) and
of the sphere geometry (camr_b200/eb_geometry.py).

* geometry: fluid volume equals the exact volume outside the sphere;
  regular cells have all faces open; covered cells none;
* mass and energy of one EB hydro evaluation on a periodic domain with a
  sphere sum to zero (the wall flux carries no mass or energy), with and
  without flux redistribution;
* with the sphere far outside the box every cell is regular and the EB path
  agrees with the regular MOL path to round-off.
"""
import os

import numpy as np
import pytest

import oracle
from camr_b200 import eb_geometry as E
from camr_b200 import problems as P

HAVE_EB = os.path.exists(oracle.lib_path_eb())
needs_eb = pytest.mark.skipif(not HAVE_EB, reason="oracle/_ref EB library not built")

N = 20


def periodic_case(seed=3, radius=0.2):
    n = (N, N, N)
    dx = 1.0 / N
    geo = E.sphere_geometry((-5, -5, -5), (N + 4, N + 4, N + 4), dx, radius=radius)
    s = P.random_smooth(n, seed=seed, amp=0.1, vel=0.2)
    p = oracle.default_params(do_mol=1, cfl=0.3)
    lev = oracle.make_level(n)
    oracle.init_finalize("restate", p, lev, s)
    G = np.pad(s, ((0, 0), (5, 5), (5, 5), (5, 5)), mode="wrap")
    return p, geo, G, dx


def test_sphere_geometry_moments():
    dx = 1.0 / 32
    geo = E.sphere_geometry((0, 0, 0), (31, 31, 31), dx, radius=0.25)
    vol = geo["vfrac"].sum() * dx ** 3
    assert abs(vol - (1.0 - 4.0 / 3.0 * np.pi * 0.25 ** 3)) < 2e-5
    typ = geo["flag"] & 3
    for d in range(3):
        ax = 2 - d
        a = geo["ap"][d]
        s0 = [slice(None)] * 3
        s1 = [slice(None)] * 3
        s0[ax] = slice(0, -1)
        s1[ax] = slice(1, None)
        lo, hi = a[tuple(s0)], a[tuple(s1)]
        assert np.all(lo[typ == 0] == 1.0) and np.all(hi[typ == 0] == 1.0)
        assert np.all(lo[typ == 3] == 0.0) and np.all(hi[typ == 3] == 0.0)
    assert ((typ == 1).sum() > 0) and ((typ == 3).sum() > 0)


@needs_eb
@pytest.mark.parametrize("redist", [0, 1])
def test_eb_hydro_conserves_mass_and_energy(redist):
    p, geo, G, dx = periodic_case()
    d, _, nass = oracle.hydro_box_eb(p, (0, 0, 0), (N - 1,) * 3, (0, 0, 0), (N - 1,) * 3,
                                     (0, 0, 0), (0, 0, 0), (1, 1, 1), G, (-5, -5, -5), geo,
                                     (dx,) * 3, 1e-3, redist=redist)
    assert nass == 0 and np.isfinite(d).all()
    vf = geo["vfrac"][5:-5, 5:-5, 5:-5]
    for c, scale in ((P.URHO, 1.0), (P.UEDEN, 10.0), (P.UFS, 1.0)):
        tot = (vf * d[c]).sum() * dx ** 3
        ref = (vf * np.abs(d[c])).sum() * dx ** 3
        assert abs(tot) <= 1e-13 * ref, (c, tot, ref)


@needs_eb
def test_eb_path_without_cut_cells_matches_regular_path():
    p, _, G, dx = periodic_case(seed=4)
    geo = E.sphere_geometry((-5, -5, -5), (N + 4,) * 3, dx, center=(9.0, 9.0, 9.0), radius=0.1)
    assert np.all((geo["flag"] & 3) == 0)
    d, _, _ = oracle.hydro_box_eb(p, (0, 0, 0), (N - 1,) * 3, (0, 0, 0), (N - 1,) * 3,
                                  (0, 0, 0), (0, 0, 0), (1, 1, 1), G, (-5, -5, -5), geo,
                                  (dx,) * 3, 1e-3, redist=1)
    r, _, _ = oracle.hydro_box("restate", p, [0, 0, 0], [N - 1] * 3, [0, 0, 0], [N - 1] * 3,
                               [0, 0, 0], [0, 0, 0], G[:, 1:-1, 1:-1, 1:-1], [-4, -4, -4],
                               (dx,) * 3, 1e-3)
    for c in (0, 1, 2, 3, 4, 5, 7, 8, 9):
        rel = np.abs(d[c] - r[c]).max() / max(np.abs(r[c]).max(), 1e-300)
        assert rel < 1e-11, (c, rel)


def eb_level_case(kind, n=(16, 16, 16), seed=5, radius=None, max_grid_size=(0, 0, 0),
                  do_mol=1):
    """(params, level, geometry over grow(domain, ng), initial state) of the
    EB level step: 'periodic' (random smooth flow around a sphere in a
    periodic cube) or 'sod' (Sod + sphere on [0,2]x[0,1]^2, x outflow, y/z
    slip walls).  max_grid_size chops the domain into boxes (0: one box).
    do_mol = 0: Godunov PLM (ng = 6 ghost cells instead of 5)."""
    ng = 5 if do_mol else 6
    glo = (-ng,) * 3
    if kind == "periodic":
        dx = 1.0 / n[0]
        geo = E.sphere_geometry(glo, tuple(v + ng - 1 for v in n), dx,
                                radius=radius or 0.2)
        s = P.random_smooth(n, seed=seed, amp=0.1, vel=0.2)
        lev = oracle.make_level(n, dx=(dx,) * 3, max_grid_size=max_grid_size)
    else:
        dx = 2.0 / n[0]
        geo = E.sphere_geometry(glo, tuple(v + ng - 1 for v in n), dx,
                                center=(1.0, 0.5, 0.5), radius=radius or 0.15)
        s = P.sod_sphere(n, (dx,) * 3, geo)
        lev = oracle.make_level(n, periodic=(0, 0, 0), bc_lo=(2, 4, 4), bc_hi=(2, 4, 4),
                                dx=(dx,) * 3, max_grid_size=max_grid_size)
    E.set_covered(s, geo)
    p = oracle.default_params(do_mol=do_mol, ppm_type=0, cfl=0.3)
    s = np.ascontiguousarray(s)
    oracle.eb_init_finalize(p, lev, s)
    return p, lev, geo, s


@needs_eb
@pytest.mark.parametrize("redist", [0, 1])
def test_eb_level_conserves_mass_and_keeps_covered_cells_zero(redist):
    p, lev, geo, s = eb_level_case("periodic")
    if not redist:
        # without redistribution the tiny cut cells limit the stable step
        # to about vfrac * CFL (the reason redistribution exists)
        p.fixed_dt = 1e-4
    vf = geo["vfrac"][5:-5, 5:-5, 5:-5]
    m0 = (vf * s[P.URHO]).sum()
    e0 = (vf * s[P.UEDEN]).sum()
    dt, hist, nass = oracle.eb_advance(p, lev, geo, s, 6, redist=redist)
    assert nass == 0 and np.isfinite(s).all() and (hist > 0).all()
    m1 = (vf * s[P.URHO]).sum()
    e1 = (vf * s[P.UEDEN]).sum()
    assert abs(m1 - m0) <= 1e-13 * m0 and abs(e1 - e0) <= 1e-13 * e0
    cov = (geo["flag"][5:-5, 5:-5, 5:-5] & 3) == 3
    assert cov.any() and np.all(s[:, cov] == 0.0)
    assert np.all(s[P.URHO][~cov] > 0.0)


@needs_eb
def test_eb_level_without_cut_cells_matches_regular_level():
    n = (16, 16, 16)
    p, lev, _, _ = eb_level_case("periodic", n=n, seed=6)
    geo = E.sphere_geometry((-5, -5, -5), tuple(v + 4 for v in n), 1.0 / n[0],
                            center=(9.0, 9.0, 9.0), radius=0.1)
    assert np.all((geo["flag"] & 3) == 0)
    s = np.ascontiguousarray(P.random_smooth(n, seed=6, amp=0.1, vel=0.2))
    oracle.eb_init_finalize(p, lev, s)
    a = s.copy()
    b = s.copy()
    oracle.eb_advance(p, lev, geo, a, 4)
    oracle.advance("restate", p, lev, b, 4)
    for c in (0, 1, 2, 3, 4, 5, 6, 7):
        rel = np.abs(a[c] - b[c]).max() / max(np.abs(b[c]).max(), 1e-300)
        assert rel < 1e-11, (c, rel)


@needs_eb
def test_eb_level_sod_sphere_runs_and_holds_the_wall():
    p, lev, geo, s = eb_level_case("sod", n=(32, 16, 16))
    dt, hist, nass = oracle.eb_advance(p, lev, geo, s, 8, redist=1)
    assert nass == 0 and np.isfinite(s).all()
    cov = (geo["flag"][5:-5, 5:-5, 5:-5] & 3) == 3
    assert np.all(s[:, cov] == 0.0) and np.all(s[P.URHO][~cov] > 0.0)
    # slip walls at y and z: no mass flux through them, outflow at x only
    # changes mass through the x faces; a symmetric problem stays symmetric
    # in y and z
    assert np.abs(s[P.URHO] - s[P.URHO][:, ::-1, :]).max() < 1e-12
    assert np.abs(s[P.URHO] - s[P.URHO][::-1, :, :]).max() < 1e-12


def box_kinds(geo, n, mgs):
    """Counts of covered / all-regular (grow 2) / cut boxes of the chop."""
    typ = geo["flag"] & 3
    o = -geo["lo"][0]
    out = {"covered": 0, "regular": 0, "cut": 0}
    for k in range(0, n[2], mgs[2]):
        for j in range(0, n[1], mgs[1]):
            for i in range(0, n[0], mgs[0]):
                b = typ[o + k:o + k + mgs[2], o + j:o + j + mgs[1], o + i:o + i + mgs[0]]
                g = typ[o - 2 + k:o + 2 + k + mgs[2], o - 2 + j:o + 2 + j + mgs[1],
                        o - 2 + i:o + 2 + i + mgs[0]]
                if np.all(b == 3):
                    out["covered"] += 1
                elif np.all(g == 0):
                    out["regular"] += 1
                else:
                    out["cut"] += 1
    return out


@needs_eb
@pytest.mark.parametrize("mgs,radius", [((8, 8, 8), 0.15), ((2, 2, 2), 0.25)])
def test_eb_level_box_decomposition(mgs, radius):
    """Regular boxes take the regular hydro, cut boxes the EB hydro, covered
    boxes none (an EB build's construct_hydro_source): the result agrees
    with the one-box EB run to round-off, conserves mass, and keeps covered
    cells zero."""
    n = (32, 16, 16)
    p, lev, geo, s = eb_level_case("sod", n=n, radius=radius, max_grid_size=mgs)
    kinds = box_kinds(geo, n, mgs)
    assert kinds["regular"] > 0 and kinds["cut"] > 0
    if mgs == (2, 2, 2):
        assert kinds["covered"] > 0
    _, lev1, _, _ = eb_level_case("sod", n=n, radius=radius)
    one = s.copy()
    a = s.copy()
    vf = geo["vfrac"][5:-5, 5:-5, 5:-5]
    nass = oracle.eb_advance(p, lev, geo, a, 5)[2]
    oracle.eb_advance(p, lev1, geo, one, 5)
    assert nass == 0 and np.isfinite(a).all()
    for c in (0, 1, 4, 5):
        rel = np.abs(a[c] - one[c]).max() / np.abs(one[c]).max()
        assert rel < 1e-10, (c, rel)
    cov = (geo["flag"][5:-5, 5:-5, 5:-5] & 3) == 3
    assert np.all(a[:, cov] == 0.0)
    # mass changes only through the outflow faces at x: compare the interior
    # mass change of both runs
    m0 = (vf * s[P.URHO]).sum()
    assert abs((vf * a[P.URHO]).sum() - (vf * one[P.URHO]).sum()) <= 1e-12 * m0


def periodic_case_ng(ng, seed=3, radius=0.2):
    n = (N, N, N)
    dx = 1.0 / N
    geo = E.sphere_geometry((-ng,) * 3, (N + ng - 1,) * 3, dx, radius=radius)
    s = P.random_smooth(n, seed=seed, amp=0.1, vel=0.2)
    p = oracle.default_params(do_mol=0, ppm_type=0, cfl=0.3)
    lev = oracle.make_level(n)
    oracle.init_finalize("restate", p, lev, s)
    G = np.pad(s, ((0, 0), (ng, ng), (ng, ng), (ng, ng)), mode="wrap")
    return p, geo, G, dx


@needs_eb
@pytest.mark.parametrize("redist", [0, 1])
def test_eb_godunov_box_conserves_mass_and_energy(redist):
    """Godunov_umeth_eb (CTU-PLM with cut cells) + the EB divergence and
    redistribution: one evaluation on a periodic domain conserves."""
    p, geo, G, dx = periodic_case_ng(6)
    d, _, nass = oracle.hydro_box_eb(p, (0, 0, 0), (N - 1,) * 3, (0, 0, 0), (N - 1,) * 3,
                                     (0, 0, 0), (0, 0, 0), (1, 1, 1), G, (-6, -6, -6), geo,
                                     (dx,) * 3, 1e-3, redist=redist)
    assert nass == 0 and np.isfinite(d).all()
    vf = geo["vfrac"][6:-6, 6:-6, 6:-6]
    for c in (P.URHO, P.UEDEN, P.UFS):
        tot = (vf * d[c]).sum() * dx ** 3
        ref = (vf * np.abs(d[c])).sum() * dx ** 3
        assert abs(tot) <= 1e-13 * ref, (c, tot, ref)


@needs_eb
def test_eb_godunov_without_cut_cells_matches_regular_ctu():
    p, _, G, dx = periodic_case_ng(6, seed=4)
    geo = E.sphere_geometry((-6, -6, -6), (N + 5,) * 3, dx, center=(9.0, 9.0, 9.0), radius=0.1)
    assert np.all((geo["flag"] & 3) == 0)
    d, _, _ = oracle.hydro_box_eb(p, (0, 0, 0), (N - 1,) * 3, (0, 0, 0), (N - 1,) * 3,
                                  (0, 0, 0), (0, 0, 0), (1, 1, 1), G, (-6, -6, -6), geo,
                                  (dx,) * 3, 1e-3, redist=1)
    r, _, _ = oracle.hydro_box("restate", p, [0, 0, 0], [N - 1] * 3, [0, 0, 0], [N - 1] * 3,
                               [0, 0, 0], [0, 0, 0], G[:, 2:-2, 2:-2, 2:-2], [-4, -4, -4],
                               (dx,) * 3, 1e-3)
    for c in (0, 1, 2, 3, 4, 5, 7, 8, 9):
        rel = np.abs(d[c] - r[c]).max() / max(np.abs(r[c]).max(), 1e-300)
        assert rel < 1e-11, (c, rel)


@needs_eb
@pytest.mark.parametrize("mgs", [(0, 0, 0), (8, 8, 8)])
def test_eb_level_godunov_sod_sphere(mgs):
    """Godunov-PLM EB level steps (6 ghost cells): finite, covered cells
    zero, the y/z mirror symmetry kept, and the box loop agrees with the
    one-box run to round-off."""
    n = (32, 16, 16)
    p, lev, geo, s = eb_level_case("sod", n=n, max_grid_size=mgs, do_mol=0)
    a = s.copy()
    _, hist, nass = oracle.eb_advance(p, lev, geo, a, 6)
    assert nass == 0 and np.isfinite(a).all() and (hist > 0).all()
    cov = (geo["flag"][6:-6, 6:-6, 6:-6] & 3) == 3
    assert np.all(a[:, cov] == 0.0) and np.all(a[P.URHO][~cov] > 0.0)
    assert np.abs(a[P.URHO] - a[P.URHO][:, ::-1, :]).max() < 1e-12
    if mgs[0]:
        _, lev1, _, _ = eb_level_case("sod", n=n, do_mol=0)
        one = s.copy()
        oracle.eb_advance(p, lev1, geo, one, 6)
        for c in (0, 1, 4, 5):
            rel = np.abs(a[c] - one[c]).max() / np.abs(one[c]).max()
            assert rel < 1e-10, (c, rel)


@needs_eb
@pytest.mark.parametrize("do_mol", [1, 0])
def test_eb_state_redistribution_conserves(do_mol):
    """State redistribution (redist = 2, one more ghost layer) conserves
    vfrac-weighted mass, energy and species in one evaluation."""
    ng = (5 if do_mol else 6) + 1
    n = (N, N, N)
    dx = 1.0 / N
    geo = E.sphere_geometry((-ng,) * 3, (N + ng - 1,) * 3, dx, radius=0.2)
    s = P.random_smooth(n, seed=3, amp=0.1, vel=0.2)
    p = oracle.default_params(do_mol=do_mol, ppm_type=0, cfl=0.3)
    lev = oracle.make_level(n)
    oracle.init_finalize("restate", p, lev, s)
    G = np.pad(s, ((0, 0), (ng, ng), (ng, ng), (ng, ng)), mode="wrap")
    d, _, nass = oracle.hydro_box_eb(p, (0, 0, 0), (N - 1,) * 3, (0, 0, 0), (N - 1,) * 3,
                                     (0, 0, 0), (0, 0, 0), (1, 1, 1), G, (-ng,) * 3, geo,
                                     (dx,) * 3, 1e-3, redist=2)
    assert nass == 0 and np.isfinite(d).all()
    vf = geo["vfrac"][ng:-ng, ng:-ng, ng:-ng]
    for c in (P.URHO, P.UEDEN, P.UFS):
        tot = (vf * d[c]).sum()
        ref = (vf * np.abs(d[c])).sum()
        assert abs(tot) <= 1e-14 * ref, (c, tot, ref)


@needs_eb
@pytest.mark.parametrize("do_mol", [1, 0])
def test_eb_state_redistribution_level_sod_sphere(do_mol):
    """Sod + sphere level steps with state redistribution and 8^3 boxes:
    finite, covered cells zero, the y/z mirror symmetry kept, and a smaller
    density undershoot near the sphere than flux redistribution gives."""
    n = (32, 16, 16)
    ng = (5 if do_mol else 6) + 1
    dx = 2.0 / n[0]
    geo = E.sphere_geometry((-ng,) * 3, tuple(v + ng - 1 for v in n), dx,
                            center=(1.0, 0.5, 0.5), radius=0.15)
    s = np.ascontiguousarray(E.set_covered(P.sod_sphere(n, (dx,) * 3, geo), geo))
    p = oracle.default_params(do_mol=do_mol, ppm_type=0, cfl=0.3)
    lev = oracle.make_level(n, periodic=(0, 0, 0), bc_lo=(2, 4, 4), bc_hi=(2, 4, 4),
                            dx=(dx,) * 3, max_grid_size=(8, 8, 8))
    oracle.eb_init_finalize(p, lev, s)
    _, hist, nass = oracle.eb_advance(p, lev, geo, s, 20, redist=2)
    assert nass == 0 and np.isfinite(s).all() and (hist > 0).all()
    cov = (geo["flag"][ng:-ng, ng:-ng, ng:-ng] & 3) == 3
    assert np.all(s[:, cov] == 0.0)
    assert np.abs(s[P.URHO] - s[P.URHO][:, ::-1, :]).max() < 1e-12
    # the same run with flux redistribution (5 / 6 ghost cells)
    ng1 = ng - 1
    geo1 = E.sphere_geometry((-ng1,) * 3, tuple(v + ng1 - 1 for v in n), dx,
                             center=(1.0, 0.5, 0.5), radius=0.15)
    f = np.ascontiguousarray(E.set_covered(P.sod_sphere(n, (dx,) * 3, geo1), geo1))
    oracle.eb_init_finalize(p, lev, f)
    oracle.eb_advance(p, lev, geo1, f, 20, redist=1)
    assert 0.125 - s[P.URHO][~cov].min() < 0.1 * (0.125 - f[P.URHO][~cov].min())
