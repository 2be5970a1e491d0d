"""GPU parity of the embedded-boundary per-box hydro (camr_hydro_umdrv_eb,
MOL) against the EB oracle (the reference's EB kernels + the restated flux
redistribution), bit for bit: a box cut by a sphere in a periodic domain,
and the Sod-with-sphere domain with outflow / slip-wall boundaries; with and
without redistribution.  Also mass and energy conservation on the device.
"""
import os

import numpy as np
import pytest

import oracle
from camr_b200 import eb_geometry as E
from camr_b200 import hydro, native
from camr_b200 import problems as P

pytestmark = pytest.mark.gpu

HAVE_EB = os.path.exists(oracle.lib_path_eb())


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def assert_bitwise(a, b, what):
    a = np.asarray(a)
    b = np.asarray(b)
    nd = int((~((a == b) | (np.isnan(a) & np.isnan(b)))).sum())
    if nd:
        rel = np.nanmax(np.abs(a - b)) / max(np.nanmax(np.abs(b)), 1e-300)
        raise AssertionError(f"{what}: {nd}/{a.size} values differ (max rel {rel:.3e})")


def periodic_case(n=24, bx=((4, 4, 4), (19, 19, 19)), seed=3, radius=0.2, ng=5):
    lo, hi = bx
    dx = 1.0 / n
    g_lo = tuple(v - ng for v in lo)
    g_hi = tuple(v + ng for v in hi)
    geo = E.sphere_geometry(g_lo, g_hi, dx, radius=radius)
    s = P.random_smooth((n, n, n), seed=seed, amp=0.1, vel=0.2)
    p = oracle.default_params(do_mol=1, cfl=0.3)
    lev = oracle.make_level((n, n, n))
    oracle.init_finalize("restate", p, lev, s)
    full = np.pad(s, ((0, 0), (ng, ng), (ng, ng), (ng, ng)), mode="wrap")  # [-ng, n+ng-1]
    sl = tuple(slice(g_lo[d] + ng, g_hi[d] + ng + 1) for d in (2, 1, 0))
    G = np.ascontiguousarray(full[(slice(None),) + sl])
    geom = hydro.make_geom((n, n, n))
    return geo, G, g_lo, lo, hi, geom, (0, 0, 0), (n - 1,) * 3, (1, 1, 1), (0, 0, 0), (0, 0, 0), dx


def sod_sphere_case(nx=32, ny=16, ng=5):
    """C4's geometry at low resolution: [0,2]x[0,1]^2, sphere r = 0.15 at
    (1, 0.5, 0.5), x outflow, y/z slip walls, Sod states (x < 0.5)."""
    dx = 1.0 / ny
    n = (nx, ny, ny)
    lo, hi = (0, 0, 0), (nx - 1, ny - 1, ny - 1)
    g_lo, g_hi = (-ng,) * 3, (nx + ng - 1, ny + ng - 1, ny + ng - 1)
    geo = E.sphere_geometry(g_lo, g_hi, dx, center=(1.0, 0.5, 0.5), radius=0.15)
    s = P.sod(n, (dx, dx, dx))
    s[P.UMX] += 0.05 * s[P.URHO]  # a little flow through the obstacle
    s[P.UEDEN] += 0.5 * 0.05 ** 2 * s[P.URHO]
    p = oracle.default_params(do_mol=1, cfl=0.3)
    lev = oracle.make_level(n, periodic=(0, 0, 0), bc_lo=(2, 4, 4), bc_hi=(2, 4, 4), dx=(dx,) * 3)
    oracle.init_finalize("restate", p, lev, s)
    G = oracle.expand_state("restate", p, lev, s, ng=ng)
    geom = hydro.make_geom(n, is_periodic=(0, 0, 0), bc_lo=(2, 4, 4), bc_hi=(2, 4, 4),
                           dx=(dx,) * 3)
    return geo, G, g_lo, lo, hi, geom, lo, hi, (0, 0, 0), (2, 4, 4), (2, 4, 4), dx


@pytest.mark.skipif(not HAVE_EB, reason="EB oracle library not built")
@pytest.mark.parametrize("case", ["periodic_box", "sod_sphere"])
@pytest.mark.parametrize("redist", [0, 1])
@pytest.mark.parametrize("do_mol", [1, 0])
def test_eb_box_matches_oracle(case, redist, do_mol):
    """MOL (MOL_umeth_eb) and Godunov-PLM (Godunov_umeth_eb) per box."""
    torch = _torch()
    ng = 5 if do_mol else 6
    geo, G, g_lo, lo, hi, geom, dlo, dhi, per, bclo, bchi, dx = (
        periodic_case(ng=ng) if case == "periodic_box" else sod_sphere_case(ng=ng))
    p = oracle.default_params(do_mol=do_mol, ppm_type=0, cfl=0.3)
    dt = 2e-3
    ref_d, ref_f, nass = oracle.hydro_box_eb(p, lo, hi, dlo, dhi, bclo, bchi, per, G, g_lo, geo,
                                             (dx,) * 3, dt, redist=redist)
    assert nass == 0
    ebdev = hydro.eb_geometry_to_device(geo)
    prm = native.default_params(do_mol=do_mol, ppm_type=0, cfl=0.3)
    d, f = hydro.hydro_umdrv_eb(lo, hi, geom, torch.from_numpy(G).cuda(), g_lo, ebdev, prm,
                                redist=bool(redist), dt=dt)
    torch.cuda.synchronize()
    assert_bitwise(d.cpu().numpy(), ref_d, "dsdt")
    for dd in range(3):
        assert_bitwise(f[dd].cpu().numpy(), ref_f[dd], f"flux {dd}")


def test_eb_box_conserves_mass_and_energy():
    torch = _torch()
    n = 24
    geo, G, g_lo, lo, hi, geom, *_rest, dx = periodic_case(n=n, bx=((0, 0, 0), (n - 1,) * 3))
    ebdev = hydro.eb_geometry_to_device(geo)
    prm = native.default_params(do_mol=1, cfl=0.3)
    d, _ = hydro.hydro_umdrv_eb(lo, hi, geom, torch.from_numpy(G).cuda(), g_lo, ebdev, prm)
    d = d.cpu().numpy()
    vf = geo["vfrac"][5:-5, 5:-5, 5:-5]
    for c in (P.URHO, P.UEDEN, P.UFS):
        tot = (vf * d[c]).sum()
        ref = (vf * np.abs(d[c])).sum()
        assert abs(tot) <= 1e-13 * ref, (c, tot, ref)


@pytest.mark.skipif(not HAVE_EB, reason="EB oracle library not built")
@pytest.mark.parametrize("kind,redist,mgs,radius,do_mol", [
    ("periodic", 1, (0, 0, 0), None, 1), ("periodic", 0, (0, 0, 0), None, 1),
    ("sod", 1, (0, 0, 0), None, 1), ("sod", 1, (8, 8, 8), 0.15, 1),
    ("sod", 1, (2, 2, 2), 0.25, 1), ("periodic", 1, (8, 8, 4), None, 1),
    ("sod", 1, (0, 0, 0), None, 0), ("sod", 1, (8, 8, 8), 0.15, 0),
    ("periodic", 1, (8, 8, 4), None, 0), ("sod", 0, (2, 2, 2), 0.25, 0)])
def test_eb_level_steps_match_oracle(kind, redist, mgs, radius, do_mol):
    """camr_eb_level_* steps (dt on the device, graph-captured after the
    first step) against the EB oracle's level driver: states and dts.  With
    a box decomposition, regular boxes run the batched regular hydro and cut
    boxes the EB hydro, covered boxes nothing."""
    _torch()
    from test_oracle_eb import eb_level_case
    n = (16, 16, 16) if kind == "periodic" else (32, 16, 16)
    p, lev, geo, s = eb_level_case(kind, n=n, radius=radius, max_grid_size=mgs, do_mol=do_mol)
    if not redist:
        p.fixed_dt = 1e-4
    ref = s.copy()
    nsteps = 6
    _, ref_dts, nass = oracle.eb_advance(p, lev, geo, ref, nsteps, redist=redist)
    assert nass == 0
    if kind == "periodic":
        geom = hydro.make_geom(n, dx=(1.0 / n[0],) * 3)
    else:
        geom = hydro.make_geom(n, is_periodic=(0, 0, 0), bc_lo=(2, 4, 4), bc_hi=(2, 4, 4),
                               dx=(2.0 / n[0],) * 3)
    prm = native.default_params(do_mol=do_mol, ppm_type=0, cfl=0.3, fixed_dt=p.fixed_dt)
    L = hydro.EBLevel(geom, prm, geo, redist=redist, max_grid_size=mgs)
    L.set_state(s)
    if mgs[0]:
        kinds = L.boxes()
        assert kinds["cut"] > 0 and (kind == "periodic" or kinds["regular"] > 0)
        # tuned launch shapes change no bits
        L.advance(2)
        L.autotune()
        L.advance(nsteps - 2)
    else:
        L.advance(nsteps)
    got = L.get_state()
    dts = L.dts()
    assert L.error()[0] == 0
    assert L.kernels_per_step() > 0
    assert_bitwise(dts, ref_dts, "dt")
    assert_bitwise(got, ref, "state")
    L.close()


def test_eb_level_init_finalize_matches_oracle():
    _torch()
    if not HAVE_EB:
        pytest.skip("EB oracle library not built")
    from test_oracle_eb import eb_level_case
    n = (32, 16, 16)
    p, lev, geo, _ = eb_level_case("sod", n=n)
    dx = 2.0 / n[0]
    raw = np.ascontiguousarray(E.set_covered(P.sod_sphere(n, (dx,) * 3, geo), geo))
    ref = raw.copy()
    oracle.eb_init_finalize(p, lev, ref)
    geom = hydro.make_geom(n, is_periodic=(0, 0, 0), bc_lo=(2, 4, 4), bc_hi=(2, 4, 4),
                           dx=(dx,) * 3)
    L = hydro.EBLevel(geom, native.default_params(do_mol=1, cfl=0.3), geo)
    L.set_state(raw)
    L.init_finalize()
    assert_bitwise(L.get_state(), ref, "state")
    L.close()


@pytest.mark.skipif(not HAVE_EB, reason="EB oracle library not built")
@pytest.mark.parametrize("case", ["periodic_box", "sod_sphere"])
@pytest.mark.parametrize("do_mol", [1, 0])
def test_eb_box_state_redistribution_matches_oracle(case, do_mol):
    """State redistribution (redist = 2) per box, bit for bit."""
    torch = _torch()
    ng = (5 if do_mol else 6) + 1
    geo, G, g_lo, lo, hi, geom, dlo, dhi, per, bclo, bchi, dx = (
        periodic_case(ng=ng) if case == "periodic_box" else sod_sphere_case(ng=ng))
    p = oracle.default_params(do_mol=do_mol, ppm_type=0, cfl=0.3)
    dt = 2e-3
    ref_d, ref_f, nass = oracle.hydro_box_eb(p, lo, hi, dlo, dhi, bclo, bchi, per, G, g_lo, geo,
                                             (dx,) * 3, dt, redist=2)
    assert nass == 0
    ebdev = hydro.eb_geometry_to_device(geo)
    prm = native.default_params(do_mol=do_mol, ppm_type=0, cfl=0.3)
    d, f = hydro.hydro_umdrv_eb(lo, hi, geom, torch.from_numpy(G).cuda(), g_lo, ebdev, prm,
                                redist=2, dt=dt)
    torch.cuda.synchronize()
    assert_bitwise(d.cpu().numpy(), ref_d, "dsdt")
    for dd in range(3):
        assert_bitwise(f[dd].cpu().numpy(), ref_f[dd], f"flux {dd}")


@pytest.mark.skipif(not HAVE_EB, reason="EB oracle library not built")
@pytest.mark.parametrize("kind,mgs,do_mol", [("sod", (8, 8, 8), 1), ("sod", (8, 8, 8), 0),
                                             ("periodic", (0, 0, 0), 1)])
def test_eb_level_state_redistribution_matches_oracle(kind, mgs, do_mol):
    """EB level steps with state redistribution against the oracle."""
    _torch()
    n = (16, 16, 16) if kind == "periodic" else (32, 16, 16)
    ng = (5 if do_mol else 6) + 1
    if kind == "periodic":
        dx = 1.0 / n[0]
        geo = E.sphere_geometry((-ng,) * 3, tuple(v + ng - 1 for v in n), dx, radius=0.2)
        s = P.random_smooth(n, seed=5, amp=0.1, vel=0.2)
        lev = oracle.make_level(n, dx=(dx,) * 3, max_grid_size=mgs)
        geom = hydro.make_geom(n, dx=(dx,) * 3)
    else:
        dx = 2.0 / n[0]
        geo = E.sphere_geometry((-ng,) * 3, tuple(v + ng - 1 for v in n), dx,
                                center=(1.0, 0.5, 0.5), radius=0.15)
        s = P.sod_sphere(n, (dx,) * 3, geo)
        lev = oracle.make_level(n, periodic=(0, 0, 0), bc_lo=(2, 4, 4), bc_hi=(2, 4, 4),
                                dx=(dx,) * 3, max_grid_size=mgs)
        geom = hydro.make_geom(n, is_periodic=(0, 0, 0), bc_lo=(2, 4, 4), bc_hi=(2, 4, 4),
                               dx=(dx,) * 3)
    s = np.ascontiguousarray(E.set_covered(s, geo))
    p = oracle.default_params(do_mol=do_mol, ppm_type=0, cfl=0.3)
    oracle.eb_init_finalize(p, lev, s)
    ref = s.copy()
    nsteps = 5
    _, ref_dts, nass = oracle.eb_advance(p, lev, geo, ref, nsteps, redist=2)
    assert nass == 0
    prm = native.default_params(do_mol=do_mol, ppm_type=0, cfl=0.3)
    L = hydro.EBLevel(geom, prm, geo, redist=2, max_grid_size=mgs)
    L.set_state(s)
    L.advance(nsteps)
    got = L.get_state()
    assert L.error()[0] == 0
    assert_bitwise(L.dts(), ref_dts, "dt")
    assert_bitwise(got, ref, "state")
    L.close()


@pytest.mark.skipif(not HAVE_EB, reason="EB oracle library not built")
@pytest.mark.parametrize("do_mol", [1, 0], ids=["mol", "godunov_plm"])
def test_eb_level_density_floor_matches_oracle(do_mol):
    """enforce_min_density on an EB level (Source/CAMR.cpp:941-1045 with the
    EB guard :960-968): an outward flow from a sphere at the centre empties
    cells below a raised small_dens; the level's boxes are the windows, covered cells
    are skipped but are neighbours.  States and dts bit for bit against the
    oracle, cells reset, error word clear."""
    _torch()
    from test_gpu_configs import evacuating_flow
    n = 24
    ng = 5 if do_mol else 6
    dx = 1.0 / n
    geo = E.sphere_geometry((-ng,) * 3, (n + ng - 1,) * 3, dx, radius=0.1)
    s = np.ascontiguousarray(E.set_covered(evacuating_flow(n, speed=1.5), geo))
    mgs = (8, 8, 8)
    p = oracle.default_params(do_mol=do_mol, ppm_type=0, cfl=0.3, small_dens=0.7)
    lev = oracle.make_level((n, n, n), dx=(dx,) * 3, max_grid_size=mgs)
    oracle.eb_init_finalize(p, lev, s)
    ref = s.copy()
    nsteps = 14
    _, ref_dts, nass = oracle.eb_advance(p, lev, geo, ref, nsteps, redist=1)
    assert nass == 0
    free = s.copy()
    p_free = oracle.default_params(do_mol=do_mol, ppm_type=0, cfl=0.3)
    oracle.eb_advance(p_free, lev, geo, free, nsteps, redist=1)
    assert not np.array_equal(free, ref)  # the floor acts
    geom = hydro.make_geom((n, n, n), dx=(dx,) * 3)
    prm = native.default_params(do_mol=do_mol, ppm_type=0, cfl=0.3, small_dens=0.7)
    L = hydro.EBLevel(geom, prm, geo, redist=1, max_grid_size=mgs)
    L.set_state(s)
    L.advance(nsteps)
    got = L.get_state()
    dts = L.dts()
    resets = L.floor_resets()
    err = L.error()
    L.close()
    assert err[0] == 0, err
    assert resets > 0
    assert_bitwise(dts, ref_dts, "dt")
    assert_bitwise(got, ref, "state")
