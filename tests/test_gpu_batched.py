"""GPU tests of the batched (work-list) hydro over uneven boxes of one level.

Every box's result must equal, bit for bit, the per-box entry point's and
the oracle's (the reference kernels when oracle/_ref is built) on the same
Sborder: batching changes the launch structure only.
"""
import numpy as np
import pytest

import oracle
from camr_b200 import problems as P

pytestmark = pytest.mark.gpu


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


# Uneven boxes inside a 40x32x24 domain (gaps allowed, no overlap).
BOXES = [((0, 0, 0), (15, 7, 11)), ((16, 0, 0), (39, 15, 7)), ((0, 8, 12), (7, 31, 23)),
         ((24, 16, 8), (39, 31, 23)), ((8, 8, 0), (23, 15, 7)), ((10, 20, 14), (13, 27, 17))]


@pytest.mark.parametrize("cfg", [dict(do_mol=0, ppm_type=1), dict(do_mol=0, ppm_type=0),
                                 dict(do_mol=1, cfl=0.3)])
def test_batched_equals_per_box_and_oracle(cfg, oracle_kind, native_lib):
    torch = _torch()
    from camr_b200 import hydro, native
    n = (40, 32, 24)
    bcs = dict(periodic=(0, 1, 0), bc_lo=(2, 0, 4), bc_hi=(3, 0, 5))
    lev = oracle.make_level(n, **bcs)
    p_or = oracle.default_params(**cfg)
    s = P.random_smooth(n, seed=17)
    oracle.init_finalize(oracle_kind, p_or, lev, s)
    border = oracle.expand_state(oracle_kind, p_or, lev, s)  # lo = -4
    dt = 0.5 * oracle.est_dt(oracle_kind, p_or, lev, s)
    geom = hydro.make_geom(n, is_periodic=bcs["periodic"], bc_lo=bcs["bc_lo"], bc_hi=bcs["bc_hi"])
    prm = native.default_params(**cfg)
    dev = torch.device("cuda:0")

    def box_inputs(lo, hi):
        sl = (slice(None), slice(lo[2], hi[2] + 9), slice(lo[1], hi[1] + 9),
              slice(lo[0], hi[0] + 9))
        uin = torch.from_numpy(np.ascontiguousarray(border[sl])).to(dev)
        nb = [hi[d] - lo[d] + 1 for d in range(3)]
        dsdt = torch.zeros((10, nb[2], nb[1], nb[0]), dtype=torch.float64, device=dev)
        flx = []
        for d in range(3):
            sh = list(nb)
            sh[d] += 1
            flx.append(torch.full((10, sh[2], sh[1], sh[0]), float("nan"), dtype=torch.float64,
                                  device=dev))
        return uin, [lo[d] - 4 for d in range(3)], dsdt, flx

    per_box = []
    for lo, hi in BOXES:
        uin, ulo, dsdt, flx = box_inputs(lo, hi)
        hydro.hydro_umdrv(list(lo), list(hi), geom, uin, ulo, dsdt, flx, prm, dt)
        per_box.append((dsdt, flx))
    torch.cuda.synchronize()

    for mode in (hydro.Batch.PERSISTENT, hydro.Batch.PER_BOX):
        items = []
        for lo, hi in BOXES:
            uin, ulo, dsdt, flx = box_inputs(lo, hi)
            items.append((list(lo), list(hi), uin, ulo, dsdt, flx))
        b = hydro.Batch(items, geom, prm)
        if mode == hydro.Batch.PERSISTENT:
            b.autotune(dt)
        b.run(dt, mode)
        torch.cuda.synchronize()
        for (lo, hi), (_, _, _, _, dsdt, flx), (d_ref, f_ref) in zip(BOXES, items, per_box):
            assert torch.equal(dsdt, d_ref), (mode, lo)
            for d in range(3):
                a, r = flx[d].cpu().numpy(), f_ref[d].cpu().numpy()
                assert ((a == r) | (np.isnan(a) & np.isnan(r))).all(), (mode, lo, d)
        b.close()

    # every launch shape: cells per block 128/256/512, one block per work
    # unit or a 7-block persistent grid that strides over many work items
    # (each block re-reads its box context on every item it takes)
    names = ["ctoprim", "flatten_divu", "trace", "flux1", "flux2", "flux3", "mol_slope",
             "mol_flux", "consup"]
    for cells in (128, 256, 512):
        for grid in (0, 7):
            items = []
            for lo, hi in BOXES:
                uin, ulo, dsdt, flx = box_inputs(lo, hi)
                items.append((list(lo), list(hi), uin, ulo, dsdt, flx))
            b = hydro.Batch(items, geom, prm)
            b.set_tuning({nm: (cells, grid) for nm in names})
            assert b.tuning() == {nm: (cells, grid) for nm in names}
            b.run(dt, hydro.Batch.PERSISTENT)
            torch.cuda.synchronize()
            for (lo, hi), (_, _, _, _, dsdt, flx), (d_ref, f_ref) in zip(BOXES, items, per_box):
                assert torch.equal(dsdt, d_ref), (cells, grid, lo)
                for d in range(3):
                    a, r = flx[d].cpu().numpy(), f_ref[d].cpu().numpy()
                    assert ((a == r) | (np.isnan(a) & np.isnan(r))).all(), (cells, grid, lo, d)
            b.close()

    # and the per-box results equal the oracle's hydro on each box
    for (lo, hi), (dsdt, flx) in zip(BOXES, per_box):
        d_o, f_o, nass = oracle.hydro_box(oracle_kind, p_or, list(lo), list(hi), [0, 0, 0],
                                          [n[0] - 1, n[1] - 1, n[2] - 1], list(lev.bc_lo),
                                          list(lev.bc_hi), border, [-4, -4, -4], list(lev.dx),
                                          dt)
        assert nass == 0
        assert np.array_equal(dsdt.cpu().numpy(), d_o)
        for d in range(3):
            assert np.array_equal(flx[d].cpu().numpy(), f_o[d])
