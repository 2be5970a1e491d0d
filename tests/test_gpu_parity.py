"""GPU parity: libcamr_b200 against the CPU oracle, bit for bit.

The oracle is the reference's own per-box hydro compiled on the CPU
(oracle/_ref) when present, else the repo's restatement (pinned to it by
tests/test_oracle.py and the golden fixtures).  The bar is exact equality of
every double; the parity tolerance (relative L1 <= 1e-12 per conserved
variable) is asserted as well so that a failure reports its size.
"""
import numpy as np
import pytest

import oracle
from camr_b200 import problems as P

pytestmark = pytest.mark.gpu

REL_L1_TOL = 1e-12

CONFIGS = {
    "ctu_ppm": dict(do_mol=0, ppm_type=1),
    "ctu_plm": dict(do_mol=0, ppm_type=0),
    "mol_plm": dict(do_mol=1, cfl=0.3),
}
BCSETS = {
    "periodic": dict(periodic=(1, 1, 1), bc_lo=(0, 0, 0), bc_hi=(0, 0, 0)),
    "walls": dict(periodic=(0, 1, 0), bc_lo=(2, 0, 4), bc_hi=(2, 0, 5)),
    "sym": dict(periodic=(0, 0, 0), bc_lo=(3, 5, 2), bc_hi=(4, 2, 3)),
    "inflow": dict(periodic=(0, 1, 0), bc_lo=(1, 0, 4), bc_hi=(2, 0, 1)),
}


def rel_l1(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    out = []
    for n in range(a.shape[0]):
        den = np.abs(b[n]).sum()
        num = np.abs(a[n] - b[n]).sum()
        out.append(num / den if den > 0 else num)
    return np.array(out)


def assert_bitwise(a, b, what):
    a = np.asarray(a)
    b = np.asarray(b)
    same = (a == b) | (np.isnan(a) & np.isnan(b))
    nd = int((~same).sum())
    if nd:
        err = rel_l1(a, b) if a.ndim == 4 else None
        raise AssertionError(f"{what}: {nd}/{a.size} values differ; per-component rel L1 {err}")


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.parametrize("cfg", list(CONFIGS))
@pytest.mark.parametrize("bcs", list(BCSETS))
def test_hydro_umdrv_box(cfg, bcs, oracle_kind, native_lib):
    """Per-box hydro (hydro_umdrv) on a ragged 13x10x9 box: fluxes and dSdt."""
    torch = _torch()
    from camr_b200 import hydro, native
    n = (13, 10, 9)
    lev = oracle.make_level(n, **BCSETS[bcs])
    p_or = oracle.default_params(**CONFIGS[cfg])
    s = P.random_smooth(n, seed=11)
    oracle.init_finalize(oracle_kind, p_or, lev, s)
    border = oracle.expand_state(oracle_kind, p_or, lev, s)
    dt = 0.5 * oracle.est_dt(oracle_kind, p_or, lev, s)
    lo = [0, 0, 0]
    hi = [n[0] - 1, n[1] - 1, n[2] - 1]
    # dsdt starts from a non-zero value to check accumulation (+=)
    base = np.full((10, n[2], n[1], n[0]), 0.25)
    dsdt_o, flx_o, nass = oracle.hydro_box(oracle_kind, p_or, lo, hi, lo, hi, list(lev.bc_lo),
                                           list(lev.bc_hi), border, [-4, -4, -4],
                                           list(lev.dx), dt, dsdt_init=base)
    assert nass == 0

    geom = hydro.make_geom(n, is_periodic=BCSETS[bcs]["periodic"], bc_lo=BCSETS[bcs]["bc_lo"],
                           bc_hi=BCSETS[bcs]["bc_hi"])
    prm = native.default_params(**CONFIGS[cfg])
    dev = torch.device("cuda:0")
    uin = torch.from_numpy(border).to(dev)
    dsdt = torch.from_numpy(base.copy()).to(dev)
    flx = []
    for d in range(3):
        sh = list(n)
        sh[d] += 1
        flx.append(torch.full((10, sh[2], sh[1], sh[0]), float("nan"), dtype=torch.float64,
                              device=dev))
    hydro.hydro_umdrv(lo, hi, geom, uin, [-4, -4, -4], dsdt, flx, prm, dt)
    torch.cuda.synchronize()
    for d in range(3):
        assert_bitwise(flx[d].cpu().numpy(), flx_o[d], f"flux {d}")
    assert_bitwise(dsdt.cpu().numpy(), dsdt_o, "dsdt")


@pytest.mark.parametrize("cfg", list(CONFIGS))
def test_hydro_umdrv_subbox(cfg, oracle_kind, native_lib):
    """Per-box hydro on a 13x10x9 box inside a 24x20x18 domain whose index
    space starts at (-3, 2, 0): the box touches only the z-low wall, so the
    other faces read ghost cells that are interior cells of the level."""
    torch = _torch()
    from camr_b200 import hydro, native
    n = (24, 20, 18)
    dlo = (-3, 2, 0)
    bcs = dict(periodic=(0, 1, 0), bc_lo=(1, 0, 4), bc_hi=(2, 0, 5))
    lev = oracle.make_level(n, lo=dlo, **bcs)
    p_or = oracle.default_params(**CONFIGS[cfg])
    s = P.random_smooth(n, seed=23)
    oracle.init_finalize(oracle_kind, p_or, lev, s)
    border = oracle.expand_state(oracle_kind, p_or, lev, s)
    uin_lo = [dlo[d] - 4 for d in range(3)]
    dt = 0.5 * oracle.est_dt(oracle_kind, p_or, lev, s)
    lo = [2, 5, 0]
    hi = [14, 14, 8]
    nb = [hi[d] - lo[d] + 1 for d in range(3)]
    dsdt_o, flx_o, nass = oracle.hydro_box(oracle_kind, p_or, lo, hi, list(dlo),
                                           [dlo[d] + n[d] - 1 for d in range(3)],
                                           list(lev.bc_lo), list(lev.bc_hi), border, uin_lo,
                                           list(lev.dx), dt)
    assert nass == 0

    geom = hydro.make_geom(n, dom_lo=dlo, is_periodic=bcs["periodic"], bc_lo=bcs["bc_lo"],
                           bc_hi=bcs["bc_hi"], dx=tuple(lev.dx))
    prm = native.default_params(**CONFIGS[cfg])
    dev = torch.device("cuda:0")
    uin = torch.from_numpy(border).to(dev)
    dsdt = torch.zeros((10, nb[2], nb[1], nb[0]), dtype=torch.float64, device=dev)
    flx = []
    for d in range(3):
        sh = list(nb)
        sh[d] += 1
        flx.append(torch.full((10, sh[2], sh[1], sh[0]), float("nan"), dtype=torch.float64,
                              device=dev))
    hydro.hydro_umdrv(lo, hi, geom, uin, uin_lo, dsdt, flx, prm, dt)
    torch.cuda.synchronize()
    for d in range(3):
        assert_bitwise(flx[d].cpu().numpy(), flx_o[d], f"flux {d}")
    assert_bitwise(dsdt.cpu().numpy(), dsdt_o, "dsdt")


def _level_run(kind, cfg, n, bcs, state0, nsteps, use_graph=True, max_grid=(0, 0, 0)):
    from camr_b200 import hydro, native
    p_or = oracle.default_params(**cfg)
    lev = oracle.make_level(n, **bcs)
    s_or = state0.copy()
    oracle.init_finalize(kind, p_or, lev, s_or)
    _, hist_or, nass = oracle.advance(kind, p_or, lev, s_or, nsteps)
    assert nass == 0

    geom = hydro.make_geom(n, is_periodic=bcs["periodic"], bc_lo=bcs["bc_lo"], bc_hi=bcs["bc_hi"])
    prm = native.default_params(**cfg)
    L = hydro.Level(geom, prm, max_grid_size=max_grid, use_graph=use_graph)
    L.set_state(state0)
    L.init_finalize()
    L.advance(nsteps)
    s_gpu = L.get_state()
    dt_last = L.last_dt()
    err = L.error()
    L.close()
    return s_or, hist_or, s_gpu, dt_last, err


@pytest.mark.parametrize("graph", [True, False])
def test_level_sod_ctu_plm(graph, oracle_kind, native_lib):
    """Config-0 shape at reduced size: Sod, outflow x / periodic y,z, CTU-PLM, CFL 0.8."""
    _torch()
    n = (32, 16, 16)
    dx = (1.0 / n[0], 1.0 / n[1], 1.0 / n[2])
    s0 = P.sod(n, dx)
    bcs = dict(periodic=(0, 1, 1), bc_lo=(2, 0, 0), bc_hi=(2, 0, 0))
    s_or, hist, s_gpu, dt_last, err = _level_run(oracle_kind, dict(do_mol=0, ppm_type=0, cfl=0.8),
                                                 n, bcs, s0, 12, use_graph=graph)
    assert err[0] == 0, err
    assert dt_last == hist[-1]
    assert np.all(rel_l1(s_gpu, s_or) <= REL_L1_TOL)
    assert_bitwise(s_gpu, s_or, "state")


def test_level_blobs_ctu_ppm(oracle_kind, native_lib):
    """Config-1 shape at reduced size: periodic blobs, CTU-PPM, CFL 0.7."""
    _torch()
    n = (24, 24, 24)
    dx = tuple(1.0 / v for v in n)
    s0 = P.blobs(n, dx, nblobs=6, seed=1, r_min=0.1, r_max=0.2)
    bcs = dict(periodic=(1, 1, 1), bc_lo=(0, 0, 0), bc_hi=(0, 0, 0))
    s_or, hist, s_gpu, dt_last, err = _level_run(oracle_kind, dict(do_mol=0, ppm_type=1, cfl=0.7),
                                                 n, bcs, s0, 8)
    assert err[0] == 0, err
    assert dt_last == hist[-1]
    assert_bitwise(s_gpu, s_or, "state")


def test_level_mol_walls(oracle_kind, native_lib):
    """MOL-PLM SSP-RK2 with walls and a random flow."""
    _torch()
    n = (20, 16, 12)
    s0 = P.random_smooth(n, seed=7)
    bcs = dict(periodic=(0, 1, 0), bc_lo=(3, 0, 4), bc_hi=(5, 0, 2))
    s_or, hist, s_gpu, dt_last, err = _level_run(oracle_kind, dict(do_mol=1, cfl=0.3), n, bcs,
                                                 s0, 6)
    assert err[0] == 0, err
    assert dt_last == hist[-1]
    assert_bitwise(s_gpu, s_or, "state")


@pytest.mark.parametrize("cfg", ["ctu_ppm", "mol_plm"])
def test_level_inflow(cfg, oracle_kind, native_lib):
    """Level steps with an inflow face (ghosts copy the boundary cell, as the
    Sod problem's bcnormal does), outflow opposite, a slip and a no-slip
    wall in z, and 4^3-ish boxes of max_grid_size 8."""
    _torch()
    n = (20, 12, 16)
    s0 = P.random_smooth(n, seed=5)
    bcs = dict(periodic=(0, 1, 0), bc_lo=(1, 0, 4), bc_hi=(2, 0, 5))
    s_or, hist, s_gpu, dt_last, err = _level_run(oracle_kind, CONFIGS[cfg], n, bcs, s0, 6,
                                                 max_grid=(8, 8, 8))
    assert err[0] == 0, err
    assert dt_last == hist[-1]
    assert_bitwise(s_gpu, s_or, "state")


@pytest.mark.parametrize("cfg", ["ctu_ppm", "mol_plm"])
def test_conservation_periodic(cfg, native_lib):
    """Mass, momentum and energy are conserved to round-off on a periodic domain."""
    _torch()
    from camr_b200 import hydro, native
    n = (24, 20, 16)
    s0 = P.random_smooth(n, seed=5)
    geom = hydro.make_geom(n)
    prm = native.default_params(**CONFIGS[cfg])
    L = hydro.Level(geom, prm)
    L.set_state(s0)
    L.init_finalize()
    a = L.get_state()
    L.advance(10)
    b = L.get_state()
    L.close()
    for comp in (0, 1, 2, 3, 4):
        ta = a[comp].sum()
        tb = b[comp].sum()
        scale = np.abs(a[comp]).sum()
        assert abs(tb - ta) <= 1e-13 * scale * 10, (comp, ta, tb)


# ---------------------------------------------------------------------------
# Golden fixtures: digests of the reference kernels' exact output bytes.
import hashlib  # noqa: E402
import json  # noqa: E402
import os  # noqa: E402

_GDIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
with open(os.path.join(_GDIR, "golden.json")) as _f:
    _GOLDEN = json.load(_f)


def _digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("name", [k for k, v in _GOLDEN.items() if v["kind"] == "run"])
def test_level_golden(name, native_lib):
    """Whole runs on the GPU reproduce the reference kernels' digests."""
    _torch()
    from camr_b200 import hydro, native
    g = _GOLDEN[name]
    n = tuple(g["n"])
    bcs = g["bcs"]
    s0 = np.load(os.path.join(_GDIR, name + ".npz"))["state"]
    geom = hydro.make_geom(n, is_periodic=bcs["periodic"], bc_lo=bcs["bc_lo"], bc_hi=bcs["bc_hi"])
    L = hydro.Level(geom, native.default_params(**g["cfg"]))
    L.set_state(s0)
    L.init_finalize()
    L.advance(g["nsteps"])
    s = L.get_state()
    dt = L.last_dt()
    err = L.error()
    L.close()
    assert err[0] == 0, err
    assert dt == g["dt_hist"][-1]
    assert _digest(s) == g["sha256_state"], s.sum(axis=(1, 2, 3))


@pytest.mark.parametrize("name", [k for k, v in _GOLDEN.items() if v["kind"] == "box"])
def test_box_golden(name, native_lib):
    """Per-box hydro on the GPU reproduces the reference kernels' digests."""
    torch = _torch()
    from camr_b200 import hydro, native
    g = _GOLDEN[name]
    n = tuple(g["n"])
    bcs = {k: tuple(v) for k, v in g["bcs"].items()}
    s = np.load(os.path.join(_GDIR, name + ".npz"))["state"]
    p_or = oracle.default_params(**g["cfg"])
    border = oracle.expand_state("restate", p_or, oracle.make_level(n, **bcs), s)
    geom = hydro.make_geom(n, is_periodic=bcs["periodic"], bc_lo=bcs["bc_lo"], bc_hi=bcs["bc_hi"])
    dev = torch.device("cuda:0")
    dsdt = torch.zeros((10, n[2], n[1], n[0]), dtype=torch.float64, device=dev)
    flx = []
    for d in range(3):
        sh = list(n)
        sh[d] += 1
        flx.append(torch.zeros((10, sh[2], sh[1], sh[0]), dtype=torch.float64, device=dev))
    hydro.hydro_umdrv([0, 0, 0], [n[0] - 1, n[1] - 1, n[2] - 1], geom,
                      torch.from_numpy(border).to(dev), [-4, -4, -4], dsdt, flx,
                      native.default_params(**g["cfg"]), g["dt"])
    torch.cuda.synchronize()
    assert _digest(dsdt.cpu().numpy(), *[f.cpu().numpy() for f in flx]) == g["sha256_dsdt_flux"]
