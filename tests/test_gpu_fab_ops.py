"""GPU parity of the fab-level calls (camr_fill_ghosts, camr_clean_state,
camr_est_dt, camr_get_error) against the oracle's level driver, bit for bit.

The level's data is a list of boxes (the domain chopped by max_grid_size),
each a device tensor covering its box grown by the ghost width, as an AMReX
MultiFab holds it.  FillPatch + clean_state of the boxes must equal the
oracle's expand_state (Source/CAMR.cpp:1243-1262) on every cell of every
grown box, with a density floor high enough that many cells are reset; the
oracle's neighbour window is the box (tile_size 0), as in the reference's
GPU build.
"""
import numpy as np
import pytest

import oracle
from camr_b200 import hydro, native
from camr_b200 import problems as P

pytestmark = pytest.mark.gpu

BCSETS = {
    "periodic": dict(periodic=(1, 1, 1), bc_lo=(0, 0, 0), bc_hi=(0, 0, 0)),
    "walls": dict(periodic=(0, 1, 0), bc_lo=(2, 0, 4), bc_hi=(2, 0, 5)),
    "sym": dict(periodic=(0, 0, 0), bc_lo=(3, 5, 2), bc_hi=(4, 2, 3)),
    "inflow": dict(periodic=(0, 1, 0), bc_lo=(1, 0, 4), bc_hi=(2, 0, 1)),
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
    assert nd == 0, f"{what}: {nd}/{a.size} values differ"


def box_tensors(torch, s, boxes, ng, fill=np.nan):
    """Each box's grown region as a tensor: valid cells from s, ghosts `fill`."""
    out = []
    for lo, hi in boxes:
        nb = [hi[d] - lo[d] + 1 + 2 * ng for d in range(3)]
        a = np.full((10, nb[2], nb[1], nb[0]), fill)
        a[:, ng:ng + hi[2] - lo[2] + 1, ng:ng + hi[1] - lo[1] + 1, ng:ng + hi[0] - lo[0] + 1] = \
            s[:, lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1]
        out.append(torch.from_numpy(a).to("cuda:0"))
    return out


@pytest.mark.parametrize("bcs", list(BCSETS))
def test_fill_ghosts_and_clean_state_match_expand_state(bcs, oracle_kind, native_lib):
    torch = _torch()
    n = (20, 16, 12)
    mgs = (8, 8, 6)
    ng = 4
    cfg = dict(do_mol=0, ppm_type=1, small_dens=0.95)
    s = P.random_smooth(n, seed=13)
    p = oracle.default_params(**cfg)
    lev = oracle.make_level(n, max_grid_size=mgs, **BCSETS[bcs])
    oracle.init_finalize(oracle_kind, oracle.default_params(do_mol=0), lev, s)
    assert (s[P.URHO] < 0.95).sum() > 100  # the floor resets many cells
    border = oracle.expand_state(oracle_kind, p, lev, s, ng=ng)
    geom = hydro.make_geom(n, is_periodic=BCSETS[bcs]["periodic"], bc_lo=BCSETS[bcs]["bc_lo"],
                           bc_hi=BCSETS[bcs]["bc_hi"])
    boxes = hydro.level_boxes(n, mgs)
    ts = box_tensors(torch, s, boxes, ng)
    hydro.fill_ghosts(geom, boxes, ts, ng)
    hydro.clean_state(geom, boxes, ts, ng, native.default_params(**cfg))
    torch.cuda.synchronize()
    assert hydro.get_error()[0] == 0
    for (lo, hi), t in zip(boxes, ts):
        want = border[:, lo[2]:hi[2] + 1 + 2 * ng, lo[1]:hi[1] + 1 + 2 * ng,
                      lo[0]:hi[0] + 1 + 2 * ng]
        assert_bitwise(t.cpu().numpy(), want, f"box {lo}-{hi}")


@pytest.mark.parametrize("n,mgs,frac", [((16, 16, 16), (8, 8, 8), None),
                                        ((32, 32, 32), (16, 16, 16), 0.3)],
                         ids=["small", "many_below_floor"])
def test_clean_state_valid_cells_match_oracle(n, mgs, frac, oracle_kind, native_lib):
    """clean_state of a MultiFab without ghost cells (the reference's
    clean_state(S_old) at the start of CAMR_advance).  many_below_floor: the
    floor is the density's 30th percentile, ~9800 cells below it in one
    pass (more than 4096: the fixup's list and its shared-memory sort hold
    16384)."""
    torch = _torch()
    s = P.random_smooth(n, seed=29)
    small = 0.9 if frac is None else float(np.quantile(s[P.URHO], frac))
    cfg = dict(do_mol=1, cfl=0.3, small_dens=small)
    if frac is not None:
        assert (s[P.URHO] < small).sum() > 4096
    lev = oracle.make_level(n, max_grid_size=mgs)
    ref = s.copy()
    oracle.clean_state(oracle_kind, oracle.default_params(**cfg), lev, ref)
    geom = hydro.make_geom(n)
    boxes = hydro.level_boxes(n, mgs)
    ts = box_tensors(torch, s, boxes, 0)
    hydro.clean_state(geom, boxes, ts, 0, native.default_params(**cfg))
    torch.cuda.synchronize()
    got = np.zeros_like(s)
    for (lo, hi), t in zip(boxes, ts):
        got[:, lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1] = t.cpu().numpy()
    assert not np.array_equal(got, s)
    assert_bitwise(got, ref, "state")


@pytest.mark.parametrize("fixed_dt", [-1.0, 2.5e-3])
def test_est_dt_matches_oracle(fixed_dt, oracle_kind, native_lib):
    torch = _torch()
    n = (24, 12, 20)
    cfg = dict(do_mol=0, ppm_type=0, cfl=0.8, fixed_dt=fixed_dt)
    s = P.blobs(n, tuple(1.0 / v for v in n), nblobs=4, seed=2, r_min=0.1, r_max=0.2,
                vel=(0.5, -0.2, 0.1))
    lev = oracle.make_level(n)
    p = oracle.default_params(**cfg)
    oracle.init_finalize(oracle_kind, p, lev, s)
    want = oracle.est_dt(oracle_kind, p, lev, s)
    boxes = hydro.level_boxes(n, (8, 8, 8))
    ts = box_tensors(torch, s, boxes, 0)
    got = hydro.est_dt(hydro.make_geom(n), boxes, ts, 0, native.default_params(**cfg))
    assert got == want


def test_get_error_reports_ctoprim_failure(native_lib):
    """A negative density reaches ctoprim: the reference asserts
    (Hydro_ctoprim.H:56); the library records the cell in its error word."""
    torch = _torch()
    n = (8, 8, 8)
    geom = hydro.make_geom(n)
    s = P.random_smooth(n, seed=3)
    border = np.pad(s, ((0, 0), (4, 4), (4, 4), (4, 4)), mode="wrap")
    border[P.URHO, 4 + 2, 4 + 3, 4 + 5] = -1.0  # cell (5, 3, 2)
    dev = torch.device("cuda:0")
    uin = torch.from_numpy(np.ascontiguousarray(border)).to(dev)
    dsdt = torch.zeros((10, 8, 8, 8), dtype=torch.float64, device=dev)
    flx = [torch.zeros((10, 8 + (d == 2), 8 + (d == 1), 8 + (d == 0)), dtype=torch.float64,
                       device=dev) for d in range(3)]
    hydro.get_error()  # read and clear what earlier work left
    hydro.hydro_umdrv([0, 0, 0], [7, 7, 7], geom, uin, [-4, -4, -4], dsdt, flx,
                      native.default_params(do_mol=1, cfl=0.3), 1e-3)
    code, i, j, k = hydro.get_error()
    assert code == 1 and (i, j, k) == (5, 3, 2)
    assert hydro.get_error()[0] == 0  # read and cleared


@pytest.mark.parametrize("cfg,with_src", [(dict(do_mol=0, ppm_type=1), True),
                                          (dict(do_mol=0, ppm_type=0, use_pslope=1), True),
                                          (dict(do_mol=1, cfl=0.3), False)],
                         ids=["ctu_ppm_src", "ctu_plm_pslope_src", "mol_plm"])
def test_hydro_umdrv_full_matches_reference(cfg, with_src, native_lib):
    """camr_hydro_umdrv_full: q / qaux / src_q from the reference's own
    ctoprim and srctoprim, non-uniform face areas and cell volumes (as a
    mapped grid would give), against the reference's hydro_umdrv called with
    the same arrays (Source/Hydro/Hydro.H:11-35), bit for bit."""
    torch = _torch()
    import os
    if not os.path.exists(oracle.lib_path("ref")):
        pytest.skip("oracle/_ref not built")
    n = (14, 11, 9)
    bcs = BCSETS["walls"]
    p = oracle.default_params(**cfg)
    lev = oracle.make_level(n, **bcs)
    s = P.random_smooth(n, seed=41)
    oracle.init_finalize("ref", p, lev, s)
    border = oracle.expand_state("ref", p, lev, s)
    rng = np.random.default_rng(12)
    src = rng.standard_normal(border.shape) * 0.2 if with_src else None
    dt = 0.4 * oracle.est_dt("ref", p, lev, s)
    lo, hi = [0, 0, 0], [n[0] - 1, n[1] - 1, n[2] - 1]
    glo, ghi = [-4, -4, -4], [n[0] + 3, n[1] + 3, n[2] + 3]
    q, qaux, srcq = oracle.ref_ctoprim(p, glo, ghi, border, glo, src=src)
    dx = list(lev.dx)
    base = (dx[1] * dx[2], dx[0] * dx[2], dx[0] * dx[1])
    area = [base[d] * (1.0 + 0.1 * rng.random((n[2] + (d == 2), n[1] + (d == 1), n[0] + (d == 0))))
            for d in range(3)]
    vol = dx[0] * dx[1] * dx[2] * (1.0 + 0.1 * rng.random((n[2], n[1], n[0])))
    want_d, want_f, nass = oracle.ref_hydro_box_full(
        p, lo, hi, lo, hi, list(lev.bc_lo), list(lev.bc_hi), border, glo, q, qaux,
        srcq if with_src else None, area, vol, dx, dt)
    assert nass == 0
    dev = torch.device("cuda:0")
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    dsdt = torch.zeros((10, n[2], n[1], n[0]), dtype=torch.float64, device=dev)
    flx = [torch.full((10, n[2] + (d == 2), n[1] + (d == 1), n[0] + (d == 0)), np.nan,
                      dtype=torch.float64, device=dev) for d in range(3)]
    geom = hydro.make_geom(n, is_periodic=bcs["periodic"], bc_lo=bcs["bc_lo"], bc_hi=bcs["bc_hi"])
    hydro.hydro_umdrv_full(lo, hi, geom, T(border), glo, T(q), T(qaux), dsdt, flx,
                           native.default_params(**cfg), dt,
                           src_q=T(srcq) if with_src else None,
                           area=[T(a[None]) for a in area], vol=T(vol[None]))
    torch.cuda.synchronize()
    assert_bitwise(dsdt.cpu().numpy(), want_d, "dsdt")
    for d in range(3):
        assert_bitwise(flx[d].cpu().numpy(), want_f[d], f"flux {d}")
