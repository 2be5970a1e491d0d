"""GPU parity at the benchmark configurations' own sizes and step counts.

Each case runs the device path through the C ABI and the oracle (the
reference's own hydro kernels compiled on the CPU, oracle/_ref, with the
restated level driver) on the same seeded input for the configuration's
stated number of steps, and requires every double to agree.  The relative
L1 error per conserved component is computed and printed (and appended as
JSON to $CAMR_PARITY_REPORT when that is set) so that a run records the
size of any disagreement next to the 1e-12 bar.

  C0  64^3 Sod, outflow x / periodic y,z, CTU-PLM, CFL 0.8, 50 steps, one box
      (riemannus, and HLLC against the restatement: HLLC has no reference)
  C1  128^3 periodic blobs in 64^3 boxes, CTU-PPM, CFL 0.7, 50 steps (the
      256^3 configuration's box size and method on a domain the oracle
      finishes in about a minute)
  C2  two levels: base 64^3, fine boxes of 16-64 cells per side drawn from
      the configuration's size set, MOL-PLM RK2, subcycling, reflux, 5 coarse
      steps
  C3  forward of the adjoint configuration, 32^3 Gaussian random field +
      blast, MOL-PLM RK2, CFL 0.3, 200 steps
  C4  Sod + sphere on 64x32x32 (dx = 1/32), 16^3 boxes, MOL-PLM with flux
      redistribution and Godunov-PLM, 150 steps
"""
import json
import os

import numpy as np
import pytest

import oracle
from camr_b200 import hydro, native
from camr_b200 import problems as P

pytestmark = pytest.mark.gpu

REL_L1_TOL = 1e-12
HAVE_EB = os.path.exists(oracle.lib_path_eb())


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def rel_l1(a, b):
    a = np.asarray(a, dtype=np.float64).reshape(10, -1)
    b = np.asarray(b, dtype=np.float64).reshape(10, -1)
    out = []
    for n in range(10):
        den = np.abs(b[n]).sum()
        num = np.abs(a[n] - b[n]).sum()
        out.append(float(num / den) if den > 0 else float(num))
    return out


def report(name, got, want, steps, extra=None):
    """Print (and optionally record) the per-component relative L1 error,
    then require bit-for-bit equality."""
    got = np.asarray(got)
    want = np.asarray(want)
    err = rel_l1(got, want)
    nd = int((~((got == want) | (np.isnan(got) & np.isnan(want)))).sum())
    rec = {"case": name, "steps": steps, "values": int(want.size), "differ": nd,
           "rel_l1": err}
    if extra:
        rec.update(extra)
    print(json.dumps(rec))
    path = os.environ.get("CAMR_PARITY_REPORT")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(rec) + "\n")
    assert max(err) <= REL_L1_TOL, rec
    assert nd == 0, rec


# The oracle runs the reference's OpenMP hydro tiles (Source/CAMR.cpp:29-30)
# so that a one-box domain still uses every host thread; a level step gives
# the same bits for any tile decomposition (tests/test_oracle.py).
TILE = (1024, 16, 16)


def level_parity(kind, cfg, n, bcs, s0, nsteps, max_grid=(0, 0, 0), dx=None):
    p = oracle.default_params(**cfg)
    lev = oracle.make_level(n, max_grid_size=max_grid, tile_size=TILE, dx=dx, **bcs)
    ref = s0.copy()
    oracle.init_finalize(kind, p, lev, ref)
    _, hist, nass = oracle.advance(kind, p, lev, ref, nsteps)
    assert nass == 0
    geom = hydro.make_geom(n, is_periodic=bcs["periodic"], bc_lo=bcs["bc_lo"],
                           bc_hi=bcs["bc_hi"], dx=tuple(lev.dx))
    L = hydro.Level(geom, native.default_params(**cfg), max_grid_size=max_grid, use_graph=True)
    L.set_state(s0)
    L.init_finalize()
    L.advance(nsteps)
    got = L.get_state()
    dts = L.dt_history(nsteps) if hasattr(L, "dt_history") else None
    dt_last = L.last_dt()
    err = L.error()
    L.close()
    assert err[0] == 0, err
    assert dt_last == hist[-1]
    if dts is not None:
        assert np.array_equal(np.asarray(dts), hist)
    return got, ref


SOD_BCS = dict(periodic=(0, 1, 1), bc_lo=(2, 0, 0), bc_hi=(2, 0, 0))
PERIODIC = dict(periodic=(1, 1, 1), bc_lo=(0, 0, 0), bc_hi=(0, 0, 0))


def test_c0_sod_ctu_plm_64cube_50_steps(oracle_kind, native_lib):
    _torch()
    n = (64, 64, 64)
    s0 = P.sod(n, tuple(1.0 / v for v in n))
    got, ref = level_parity(oracle_kind, dict(do_mol=0, ppm_type=0, cfl=0.8), n, SOD_BCS, s0, 50)
    report("c0 sod 64^3 CTU-PLM riemannus", got, ref, 50, {"oracle": oracle_kind})


def test_c0_sod_ctu_plm_hllc_64cube_50_steps(native_lib):
    """The configuration's HLLC solver: no reference counterpart, so the
    oracle is the restatement (oracle/hydro_restate.cpp hllc)."""
    _torch()
    if not os.path.exists(oracle.lib_path("restate")):
        oracle.build(ref=False)
    n = (64, 64, 64)
    s0 = P.sod(n, tuple(1.0 / v for v in n))
    got, ref = level_parity("restate", dict(do_mol=0, ppm_type=0, cfl=0.8, riemann_solver=1), n,
                            SOD_BCS, s0, 50)
    report("c0 sod 64^3 CTU-PLM HLLC", got, ref, 50, {"oracle": "restate"})


def test_c1_blobs_ctu_ppm_64cube_boxes_50_steps(oracle_kind, native_lib):
    _torch()
    n = (128, 128, 128)
    s0 = P.blobs(n, tuple(1.0 / v for v in n), nblobs=16, seed=1)
    got, ref = level_parity(oracle_kind, dict(do_mol=0, ppm_type=1, cfl=0.7), n, PERIODIC, s0, 50,
                            max_grid=(64, 64, 64))
    report("c1 blobs 128^3 (8 x 64^3 boxes) CTU-PPM", got, ref, 50, {"oracle": oracle_kind})


def test_c3_forward_mol_plm_32cube_200_steps(oracle_kind, native_lib):
    _torch()
    n = (32, 32, 32)
    s0, _ = P.grf_blast(n, seed=3)
    got, ref = level_parity(oracle_kind, dict(do_mol=1, cfl=0.3), n, PERIODIC, s0, 200)
    report("c3 forward 32^3 MOL-PLM", got, ref, 200, {"oracle": oracle_kind})


def test_c2_two_level_mol_plm_5_coarse_steps(oracle_kind, native_lib):
    _torch()
    n0 = (64, 64, 64)
    boxes = P.amr_box_list(nbox=40, fine_n=128, sizes=(16, 24, 32, 48, 64), seed=7, align=8)
    cells = sum((h[0] - l[0] + 1) * (h[1] - l[1] + 1) * (h[2] - l[2] + 1) for l, h in boxes)
    assert len(boxes) >= 10
    S0, S1 = P.amr_initial(n0, boxes, nblobs=16, seed=1)
    cfg = dict(do_mol=1, ppm_type=0, cfl=0.3)
    p = oracle.default_params(**cfg)
    lev = oracle.make_level(n0)
    bx = np.array([list(lo) + list(hi) for lo, hi in boxes], dtype=np.int32)
    o0, o1 = S0.copy(), S1.copy()
    clock = np.zeros(4)
    oracle.amr_run(oracle_kind, p, lev, bx, o0, o1, 0, do_init=True, clock=clock)
    _, nerr = oracle.amr_run(oracle_kind, p, lev, bx, o0, o1, 5, first_step=True, clock=clock)
    assert nerr == 0
    h = hydro.AmrHierarchy(hydro.make_geom(n0), native.default_params(**cfg), boxes,
                           use_graph=True)
    h.set_state(S0, S1)
    h.init_finalize()
    h.advance(5)
    g0, g1 = h.get_state()
    gclock = h.clock()
    assert h.error()[0] == 0
    h.close()
    assert np.array_equal(np.asarray(gclock), clock)
    report("c2 two-level base 64^3 MOL-PLM: level 0", g0, o0, 5,
           {"oracle": oracle_kind, "fine_boxes": len(boxes), "fine_cells": cells})
    report("c2 two-level base 64^3 MOL-PLM: level 1", g1, o1, 5,
           {"oracle": oracle_kind, "fine_boxes": len(boxes), "fine_cells": cells})


@pytest.mark.skipif(not HAVE_EB, reason="EB oracle library not built")
@pytest.mark.parametrize("do_mol", [1, 0])
def test_c4_sod_sphere_64x32x32_150_steps(do_mol):
    _torch()
    from test_oracle_eb import eb_level_case
    n = (64, 32, 32)
    mgs = (16, 16, 16)
    p, lev, geo, s = eb_level_case("sod", n=n, max_grid_size=mgs, do_mol=do_mol)
    ref = s.copy()
    nsteps = 150
    _, ref_dts, nass = oracle.eb_advance(p, lev, geo, ref, nsteps, redist=1)
    assert nass == 0
    geom = hydro.make_geom(n, is_periodic=(0, 0, 0), bc_lo=(2, 4, 4), bc_hi=(2, 4, 4),
                           dx=(2.0 / n[0],) * 3)
    prm = native.default_params(do_mol=do_mol, ppm_type=0, cfl=0.3)
    L = hydro.EBLevel(geom, prm, geo, redist=1, max_grid_size=mgs)
    L.set_state(s)
    kinds = L.boxes()
    L.advance(nsteps)
    got = L.get_state()
    dts = L.dts()
    assert L.error()[0] == 0
    L.close()
    assert np.array_equal(np.asarray(dts), ref_dts)
    report(f"c4 sod+sphere 64x32x32 {'MOL' if do_mol else 'Godunov'}-PLM FluxRedist", got, ref,
           nsteps, {"oracle": "ref (EB kernels) + restated redistribution", "boxes": kinds})


@pytest.mark.parametrize("ppm_type,pslope", [(0, 0), (1, 0), (0, 1)])
def test_hydro_umdrv_with_nonzero_sources(ppm_type, pslope, oracle_kind, native_lib):
    """The per-box CTU hydro with a non-zero source fab: hydro_srctoprim
    (Hydro_ctoprim.H:106-157) feeds the primitive sources into the
    transverse (transdd) corrections and, with use_pslope = 1, into the
    pressure slope of plm_pslope (PLM.H:84-165)."""
    torch = _torch()
    n = (20, 16, 12)
    bcs = dict(periodic=(0, 1, 0), bc_lo=(2, 0, 4), bc_hi=(2, 0, 3))
    cfg = dict(do_mol=0, ppm_type=ppm_type, use_pslope=pslope)
    p_or = oracle.default_params(**cfg)
    lev = oracle.make_level(n, **bcs)
    s = P.random_smooth(n, seed=31)
    oracle.init_finalize(oracle_kind, p_or, lev, s)
    border = oracle.expand_state(oracle_kind, p_or, lev, s)
    rng = np.random.default_rng(9)
    src = rng.standard_normal(border.shape) * 0.3
    dt = 0.5 * oracle.est_dt(oracle_kind, p_or, lev, s)
    lo, hi = [0, 0, 0], [n[0] - 1, n[1] - 1, n[2] - 1]
    dsdt_o, flx_o, nass = oracle.hydro_box(oracle_kind, p_or, lo, hi, lo, hi, list(lev.bc_lo),
                                           list(lev.bc_hi), border, [-4, -4, -4], list(lev.dx),
                                           dt, src=src)
    assert nass == 0
    geom = hydro.make_geom(n, is_periodic=bcs["periodic"], bc_lo=bcs["bc_lo"],
                           bc_hi=bcs["bc_hi"])
    prm = native.default_params(**cfg)
    dev = torch.device("cuda:0")
    uin = torch.from_numpy(border).to(dev)
    srcd = torch.from_numpy(src).to(dev)
    dsdt = torch.zeros((10, n[2], n[1], n[0]), dtype=torch.float64, device=dev)
    flx = []
    for d in range(3):
        sh = list(n)
        sh[d] += 1
        flx.append(torch.zeros((10, sh[2], sh[1], sh[0]), dtype=torch.float64, device=dev))
    hydro.hydro_umdrv(lo, hi, geom, uin, [-4, -4, -4], dsdt, flx, prm, dt, src=srcd)
    torch.cuda.synchronize()
    # the sources change the result (the test would be vacuous otherwise)
    d0, _, _ = oracle.hydro_box(oracle_kind, p_or, lo, hi, lo, hi, list(lev.bc_lo),
                                list(lev.bc_hi), border, [-4, -4, -4], list(lev.dx), dt)
    assert not np.array_equal(d0, dsdt_o)
    what = f"hydro_umdrv CTU ppm_type={ppm_type} use_pslope={pslope} with sources"
    report(f"{what}: dsdt", dsdt.cpu().numpy(), dsdt_o, 1, {"oracle": oracle_kind})
    for d in range(3):
        report(f"{what}: flux {d}",
               flx[d].cpu().numpy(), flx_o[d], 1, {"oracle": oracle_kind})


@pytest.mark.parametrize("ppm_type,pslope", [(0, 0), (1, 0), (0, 1)])
def test_level_ctu_with_gravity(ppm_type, pslope, oracle_kind, native_lib):
    """CTU level steps with const_grav != 0: the old-time gravity source
    enters the hydro through sources_for_hydro -> hydro_srctoprim
    (CAMR_construct_hydro_source.cpp:28-34, 120-134), the old and new
    source Saxpys around it (CAMR_advance.cpp:110-151)."""
    _torch()
    n = (16, 16, 24)
    bcs = dict(periodic=(1, 1, 0), bc_lo=(0, 0, 4), bc_hi=(0, 0, 4))
    s0 = P.random_smooth(n, seed=17)
    cfg = dict(do_mol=0, ppm_type=ppm_type, cfl=0.6, const_grav=-2.0, use_pslope=pslope)
    got, ref = level_parity(oracle_kind, cfg, n, bcs, s0, 12)
    # gravity changed the flow (else the case would not test the sources)
    flat, _ = level_parity(oracle_kind, dict(cfg, const_grav=0.0), n, bcs, s0, 12)
    assert not np.array_equal(flat, ref)
    report(f"level CTU ppm_type={ppm_type} use_pslope={pslope} const_grav=-2", got, ref, 12,
           {"oracle": oracle_kind})


def evacuating_flow(n, seed=4, speed=3.0):
    """A smooth random density with the outward flow u = speed (x - 1/2):
    the centre empties, so cells fall below a raised density floor."""
    s = P.random_smooth((n, n, n), seed=seed, amp=0.2, vel=0.0)
    x = (np.arange(n) + 0.5) / n - 0.5
    vel = (speed * x[None, None, :], speed * x[None, :, None], speed * x[:, None, None])
    rho = s[P.URHO]
    for d in range(3):
        s[P.UMX + d] = rho * vel[d]
    s[P.UEDEN] = s[P.UEINT] + 0.5 * rho * sum(v * v for v in vel)
    return s


@pytest.mark.parametrize("cfg", [dict(do_mol=0, ppm_type=1, cfl=0.5), dict(do_mol=1, cfl=0.3)],
                         ids=["ctu_ppm", "mol_plm"])
def test_density_floor_resets_match_oracle(cfg, oracle_kind, native_lib):
    """enforce_min_density (Source/CAMR.cpp:941-1045) after the update and in
    the MOL stage-2 ghost fill: cells below small_dens take the state of the
    densest neighbour in their box or the small state, in the reference's
    sequential order, bit for bit, with the error word clear."""
    _torch()
    n = 24
    s0 = evacuating_flow(n)
    cfg = dict(cfg, small_dens=0.45)
    mgs = (8, 8, 8)
    p = oracle.default_params(**cfg)
    lev = oracle.make_level((n, n, n), max_grid_size=mgs)
    ref = s0.copy()
    oracle.init_finalize(oracle_kind, p, lev, ref)
    _, hist, nass = oracle.advance(oracle_kind, p, lev, ref, 14)
    assert nass == 0
    # the floor acts: without it the run ends elsewhere
    free = s0.copy()
    oracle.init_finalize(oracle_kind, oracle.default_params(**dict(cfg, small_dens=1e-7)), lev,
                         free)
    oracle.advance(oracle_kind, oracle.default_params(**dict(cfg, small_dens=1e-7)), lev, free, 14)
    assert not np.array_equal(free, ref)
    L = hydro.Level(hydro.make_geom((n, n, n)), native.default_params(**cfg), max_grid_size=mgs,
                    use_graph=True)
    L.set_state(s0)
    L.init_finalize()
    L.advance(14)
    got = L.get_state()
    resets = L.floor_resets()
    err = L.error()
    dt_last = L.last_dt()
    L.close()
    assert err[0] == 0, err
    assert resets > 0
    assert dt_last == hist[-1]
    assert ref[P.URHO].min() >= cfg["small_dens"]
    report(f"density floor {'MOL' if cfg['do_mol'] else 'CTU'}", got, ref, 14,
           {"oracle": oracle_kind, "cells_reset": resets})


@pytest.mark.skipif(not HAVE_EB, reason="EB oracle library not built")
def test_eb_level_godunov_pslope():
    """use_pslope = 1 on an EB Godunov-PLM level: plm_pslope_eb (PLM_eb.H:
    63-104) in the cut boxes, plm_pslope in the regular ones."""
    _torch()
    from test_oracle_eb import eb_level_case
    n = (32, 16, 16)
    mgs = (8, 8, 8)
    p, lev, geo, s = eb_level_case("sod", n=n, max_grid_size=mgs, do_mol=0)
    p.use_pslope = 1
    ref = s.copy()
    _, ref_dts, nass = oracle.eb_advance(p, lev, geo, ref, 8, redist=1)
    assert nass == 0
    geom = hydro.make_geom(n, is_periodic=(0, 0, 0), bc_lo=(2, 4, 4), bc_hi=(2, 4, 4),
                           dx=(2.0 / n[0],) * 3)
    prm = native.default_params(do_mol=0, ppm_type=0, cfl=0.3, use_pslope=1)
    L = hydro.EBLevel(geom, prm, geo, redist=1, max_grid_size=mgs)
    L.set_state(s)
    L.advance(8)
    got = L.get_state()
    dts = L.dts()
    assert L.error()[0] == 0
    L.close()
    assert np.array_equal(np.asarray(dts), ref_dts)
    report("eb level Godunov-PLM use_pslope=1", got, ref, 8, {"oracle": "ref EB kernels"})


def test_amr_ctu_plm_pslope(oracle_kind, native_lib):
    """use_pslope = 1 in the two-level driver (CTU-PLM, zero sources)."""
    _torch()
    n0 = (16, 16, 16)
    boxes = [((8, 8, 8), (15, 15, 23)), ((16, 8, 8), (23, 15, 15))]
    S0, S1 = P.amr_initial(n0, boxes, nblobs=4, r_min=0.1, r_max=0.2)
    cfg = dict(do_mol=0, ppm_type=0, cfl=0.5, use_pslope=1)
    p = oracle.default_params(**cfg)
    lev = oracle.make_level(n0)
    bx = np.array([list(lo) + list(hi) for lo, hi in boxes], dtype=np.int32)
    o0, o1 = S0.copy(), S1.copy()
    clock = np.zeros(4)
    oracle.amr_run(oracle_kind, p, lev, bx, o0, o1, 0, do_init=True, clock=clock)
    _, nerr = oracle.amr_run(oracle_kind, p, lev, bx, o0, o1, 3, first_step=True, clock=clock)
    assert nerr == 0
    h = hydro.AmrHierarchy(hydro.make_geom(n0), native.default_params(**cfg), boxes)
    h.set_state(S0, S1)
    h.init_finalize()
    h.advance(3)
    g0, g1 = h.get_state()
    assert h.error()[0] == 0
    h.close()
    report("amr CTU-PLM use_pslope=1: level 0", g0, o0, 3, {"oracle": oracle_kind})
    report("amr CTU-PLM use_pslope=1: level 1", g1, o1, 3, {"oracle": oracle_kind})
