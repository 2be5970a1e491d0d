"""GPU parity of the two-level AMR hierarchy (camr_amr_*) against the
oracle's restated two-level driver, bit for bit: subcycled steps with the
coarse-fine ghost fill (time + space interpolation), flux-register reflux,
average-down and the two-level dt control; graph replay from the second
step on.  At a larger size, total conservation on the periodic domain.
"""
import numpy as np
import pytest

import oracle
from camr_b200 import hydro, native
from camr_b200 import problems as P

pytestmark = pytest.mark.gpu

N0 = (16, 16, 16)
BOXES = [((8, 8, 8), (15, 15, 23)), ((16, 8, 8), (23, 15, 15)),
         ((0, 24, 0), (7, 31, 7)), ((24, 0, 24), (31, 7, 31))]
METHODS = {
    "mol_plm": dict(do_mol=1, ppm_type=0, cfl=0.3),
    "ctu_ppm": dict(do_mol=0, ppm_type=1, cfl=0.5),
    "ctu_plm": dict(do_mol=0, ppm_type=0, cfl=0.5),
}


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
        rel = np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)
        raise AssertionError(f"{what}: {nd}/{a.size} values differ (rel L1 {rel:.3e})")


def box_array(boxes):
    return np.array([list(lo) + list(hi) for lo, hi in boxes], dtype=np.int32)


def oracle_run(kind, method, n0, boxes, nsteps, S0, S1):
    p = oracle.default_params(**METHODS[method])
    lev = oracle.make_level(n0)
    clock = np.zeros(4)
    bx = box_array(boxes)
    oracle.amr_run(kind, p, lev, bx, S0, S1, 0, do_init=True, clock=clock)
    hist, nerr = oracle.amr_run(kind, p, lev, bx, S0, S1, nsteps, first_step=True, clock=clock)
    assert nerr == 0
    return clock


def gpu_run(method, n0, boxes, nsteps, S0, S1, use_graph=True):
    geom = hydro.make_geom(n0)
    params = native.default_params(**METHODS[method])
    h = hydro.AmrHierarchy(geom, params, boxes, use_graph=use_graph)
    h.set_state(S0, S1)
    h.init_finalize()
    h.advance(nsteps)
    a, b = h.get_state()
    clock = h.clock()
    assert h.error()[0] == 0
    h.close()
    return a, b, clock


@pytest.mark.parametrize("method", list(METHODS))
def test_amr_gpu_matches_oracle(method, oracle_kind):
    _torch()
    S0, S1 = P.amr_initial(N0, BOXES, nblobs=4, r_min=0.1, r_max=0.2)
    o0, o1 = S0.copy(), S1.copy()
    oclock = oracle_run(oracle_kind, method, N0, BOXES, 3, o0, o1)
    g0, g1, gclock = gpu_run(method, N0, BOXES, 3, S0, S1)
    assert_bitwise(gclock, oclock, "clock (times, dts)")
    assert_bitwise(g0, o0, "level 0")
    assert_bitwise(g1, o1, "level 1")


def test_amr_gpu_graph_equals_eager_and_per_box():
    _torch()
    S0, S1 = P.amr_initial(N0, BOXES, nblobs=4, r_min=0.1, r_max=0.2)
    a = gpu_run("ctu_ppm", N0, BOXES, 3, S0, S1, use_graph=True)
    b = gpu_run("ctu_ppm", N0, BOXES, 3, S0, S1, use_graph=False)
    for x, y, w in zip(a, b, ("level 0", "level 1", "clock")):
        assert_bitwise(x, y, w)
    geom = hydro.make_geom(N0)
    h = hydro.AmrHierarchy(geom, native.default_params(**METHODS["ctu_ppm"]), BOXES)
    h.set_fine_mode(h.PER_BOX)
    h.set_state(S0, S1)
    h.init_finalize()
    h.advance(3)
    c0, c1 = h.get_state()
    h.close()
    assert_bitwise(c0, a[0], "level 0 (per-box fine hydro)")
    assert_bitwise(c1, a[1], "level 1 (per-box fine hydro)")


def test_amr_gpu_larger_matches_oracle_and_conserves(oracle_kind):
    _torch()
    n0 = (48, 48, 48)
    boxes = P.amr_box_list(nbox=24, fine_n=96, sizes=(8, 16, 24), seed=3, align=8)
    S0, S1 = P.amr_initial(n0, boxes, nblobs=6, r_min=0.05, r_max=0.1)
    o0, o1 = S0.copy(), S1.copy()
    oracle_run(oracle_kind, "ctu_ppm", n0, boxes, 2, o0, o1)
    geom = hydro.make_geom(n0)
    h = hydro.AmrHierarchy(geom, native.default_params(**METHODS["ctu_ppm"]), boxes)
    h.set_state(S0, S1)
    h.init_finalize()
    start, _ = h.get_state()
    h.advance(2)
    g0, g1 = h.get_state()
    assert h.error()[0] == 0
    h.close()
    assert_bitwise(g0, o0, "level 0")
    assert_bitwise(g1, o1, "level 1")
    for comp in (P.URHO, P.UMX, P.UMY, P.UMZ, P.UEDEN):
        assert abs(start[comp].sum() - g0[comp].sum()) <= 1e-13 * np.abs(start[comp]).sum()


def inject(S0, boxes):
    """Fine box states equal to their coarse parents' (ratio 2), back to
    back in the camr_amr_set_state layout."""
    parts = []
    for lo, hi in boxes:
        sl = tuple(slice(lo[d] // 2, hi[d] // 2 + 1) for d in (2, 1, 0))
        c = S0[(slice(None),) + sl]
        parts.append(np.ascontiguousarray(c.repeat(2, 1).repeat(2, 2).repeat(2, 3)).ravel())
    return np.concatenate(parts)


@pytest.mark.parametrize("method", ["mol_plm", "ctu_ppm"])
def test_amr_density_floor_matches_oracle(method, oracle_kind):
    """enforce_min_density on both levels of the two-level step (every
    clean_state of CAMR_advance and post_timestep, Source/CAMR.cpp:941-1045):
    an outward flow empties the centre below a raised small_dens; each box
    is its own window (the base level's 8^3 boxes, each fine box), cells
    reset in the reference's order.  States and clock bit for bit against
    the oracle's two-level driver, cells reset, error word clear."""
    _torch()
    from test_gpu_configs import evacuating_flow
    n0 = (16, 16, 16)
    boxes = [((8, 8, 8), (23, 23, 23)), ((24, 0, 0), (31, 7, 15))]
    S0 = evacuating_flow(16)
    S1 = inject(S0, boxes)
    cfg = dict(METHODS[method], small_dens=0.45)
    mgs = (8, 8, 8)
    nsteps = 8
    p = oracle.default_params(**cfg)
    lev = oracle.make_level(n0, max_grid_size=mgs)
    bx = box_array(boxes)
    o0, o1 = S0.copy(), S1.copy()
    clock = np.zeros(4)
    oracle.amr_run(oracle_kind, p, lev, bx, o0, o1, 0, do_init=True, clock=clock)
    _, nerr = oracle.amr_run(oracle_kind, p, lev, bx, o0, o1, nsteps, first_step=True,
                             clock=clock)
    assert nerr == 0
    f0, f1 = S0.copy(), S1.copy()
    pf = oracle.default_params(**METHODS[method])
    cf = np.zeros(4)
    oracle.amr_run(oracle_kind, pf, lev, bx, f0, f1, 0, do_init=True, clock=cf)
    oracle.amr_run(oracle_kind, pf, lev, bx, f0, f1, nsteps, first_step=True, clock=cf)
    assert not (np.array_equal(f0, o0) and np.array_equal(f1, o1))  # the floor acts
    h = hydro.AmrHierarchy(hydro.make_geom(n0), native.default_params(**cfg), boxes,
                           max_grid_size=mgs)
    h.set_state(S0, S1)
    h.init_finalize()
    h.advance(nsteps)
    g0, g1 = h.get_state()
    gclock = h.clock()
    resets = h.floor_resets()
    err = h.error()
    h.close()
    assert err[0] == 0, err
    assert resets > 0
    assert_bitwise(gclock, clock, "clock (times, dts)")
    assert_bitwise(g0, o0, "level 0")
    assert_bitwise(g1, o1, "level 1")
