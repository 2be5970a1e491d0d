"""The two-level ghost fill across ranks (camr_b200/distributed.py
TwoLevelFill) on CPU, against the oracle's restated FillPatchTwoLevels fill
(oracle/level_driver.cpp fine_fill_boundary and cons_interp, through
orc_fine_fill_ghosts), bit for bit: fine-fine copies through the periodic
domain, the limited conservative interpolation of the coarse data, and the
time choice (old, new, or combined) of StateData::getData.  Every ghost
cell starts as NaN and must be filled."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from camr_b200 import distributed as D
from camr_b200 import hydro

N = (16, 12, 8)
MGS = (8, 6, 4)
FBOXES = [((2, 2, 2), (9, 9, 7)),       # coarse 1..4 x 1..4 x 1..3
          ((10, 2, 2), (15, 7, 5)),     # touches the first along x
          ((28, 0, 12), (31, 5, 15)),   # ghosts across the periodic x, y and z edges
          ((20, 16, 4), (21, 17, 5)),   # one coarse cell
          ((0, 18, 0), (3, 23, 1))]     # low x and high y edges
NG = 4
TIMES = {"old": (0.5, 0.75, 0.5), "new": (0.5, 0.75, 0.75), "mid": (0.5, 0.75, 0.6)}


def _inputs():
    rng = np.random.default_rng(41)
    c_old = 1.0 + 0.1 * rng.standard_normal((10,) + N[::-1])
    c_new = c_old + 0.01 * rng.standard_normal(c_old.shape)
    c_new[2, 3, 4, 5:9] = c_new[2, 3, 4, 4]      # flat runs: zero slopes
    grown = []
    for lo, hi in FBOXES:
        a = np.full((10,) + tuple(hi[e] - lo[e] + 1 + 2 * NG for e in (2, 1, 0)), np.nan)
        a[:, NG:-NG, NG:-NG, NG:-NG] = 1.0 + 0.1 * rng.standard_normal(
            (10,) + tuple(hi[e] - lo[e] + 1 for e in (2, 1, 0)))
        grown.append(a)
    return c_old, c_new, grown


def _oracle(when):
    import oracle
    c_old, c_new, grown = _inputs()
    fb = np.array([list(lo) + list(hi) for lo, hi in FBOXES])
    return oracle.fine_fill_ghosts("restate", oracle.make_level(N), fb, grown, c_old, c_new,
                                   *TIMES[when])


def _run_rank(rank, world, cowner, fowner, pg, when, device=None):
    device = device or torch.device("cpu")
    c_old, c_new, grown = _inputs()
    cboxes = hydro.level_boxes(N, MGS)
    fill = D.TwoLevelFill(hydro.make_geom(N), cboxes, cowner, FBOXES, fowner, rank, world,
                          device, pg)
    co, cn = {}, {}
    for c in fill.mine_c:
        lo, hi = cboxes[c]
        sl = (slice(None), slice(lo[2], hi[2] + 1), slice(lo[1], hi[1] + 1),
              slice(lo[0], hi[0] + 1))
        co[c] = torch.from_numpy(np.ascontiguousarray(c_old[sl])).to(device)
        cn[c] = torch.from_numpy(np.ascontiguousarray(c_new[sl])).to(device)
    fine = {b: torch.from_numpy(grown[b].copy()).to(device) for b in fill.mine_f}
    fill(fine, co, cn, *TIMES[when])
    return {b: t.cpu().numpy() for b, t in fine.items()}


def _same_bits(a, b):
    return np.array_equal(a.view(np.int64), b.view(np.int64))


@pytest.mark.parametrize("when", list(TIMES))
def test_two_level_fill_one_rank_matches_oracle(oracle_kind, when):
    want = _oracle(when)
    got = _run_rank(0, 1, [0] * len(hydro.level_boxes(N, MGS)), [0] * len(FBOXES), None, when)
    for b in range(len(FBOXES)):
        assert not np.isnan(want[b]).any()
        assert _same_bits(got[b], want[b]), b


def test_two_level_fill_time_choice():
    """getData's window: within 1e-3 (t1 - t0) of an end the end's state."""
    assert D.TwoLevelFill.time_weights(0.5, 0.75, 0.75 - 1e-5)[0] == 0
    assert D.TwoLevelFill.time_weights(0.5, 0.75, 0.5 + 1e-5)[0] == 1
    mode, a, b = D.TwoLevelFill.time_weights(0.5, 0.75, 0.6)
    assert mode == 2 and a == (0.75 - 0.6) / 0.25 and b == (0.6 - 0.5) / 0.25


def test_two_level_fill_limiter_keeps_children_in_range():
    """A coarse cell whose three slopes point the same way: the MC slopes
    are 0.2 each, the unlimited (+,+,+) child 1.15 would leave the
    neighbours' maximum 1.1, so alpha = 0.1 / 0.15 and that child lands on
    1.1 (up to rounding), the (-,-,-) child symmetrically inside."""
    import types
    v = np.ones((10, 27))
    for step in (1, 3, 9):           # x, y, z neighbours of the centre (13)
        v[:, 13 + step] = 1.1
        v[:, 13 - step] = 0.7
    cv = torch.from_numpy(v)
    inv = torch.arange(27).reshape(27, 1)
    me = types.SimpleNamespace(torch=torch)
    hi = D.TwoLevelFill._cons_interp(me, cv, inv, [torch.tensor([0.25])] * 3)
    lo = D.TwoLevelFill._cons_interp(me, cv, inv, [torch.tensor([-0.25])] * 3)
    a = 0.1 / (0.25 * 0.2 + 0.25 * 0.2 + 0.25 * 0.2)
    assert 1.0 + 0.25 * 0.2 * 3 > 1.1                   # unlimited would overshoot
    assert np.allclose(hi.numpy(), 1.0 + 3 * 0.25 * 0.2 * a, rtol=0, atol=1e-15)
    assert np.all(hi.numpy() <= 1.1 + 1e-15) and np.all(lo.numpy() >= 0.7)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, fowner, when, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cowner = D.sfc_partition(hydro.level_boxes(N, MGS), world)
        q.put((rank, _run_rank(rank, world, cowner, fowner, dist, when)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,fowner,when", [(2, [0, 1, 0, 1, 1], "mid"),
                                               (2, [1, 1, 1, 1, 1], "old"),
                                               (3, [2, 0, 1, 2, 0], "mid")])
def test_two_level_fill_several_ranks_matches_oracle(oracle_kind, world, fowner, when):
    want = _oracle(when)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, fowner, when, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got = {}
    for _, part in res:
        assert not set(part) & set(got)
        got.update(part)
    assert sorted(got) == list(range(len(FBOXES)))
    for b in range(len(FBOXES)):
        assert _same_bits(got[b], want[b]), b
