"""The box-distributed level (camr_b200/distributed.py) on CPU: the
space-filling-curve partition, and the ghost-cell exchange over two gloo
processes against an independent fill of the whole domain (periodic wrap,
and past physical boundaries the BC map: foextrap / ext_dir copy the edge,
reflect_even / reflect_odd mirror it, odd components change sign), plus
the dt minimum over the ranks."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from camr_b200 import distributed as D
from camr_b200 import hydro

BCSETS = {
    "periodic": dict(is_periodic=(1, 1, 1), bc_lo=(0, 0, 0), bc_hi=(0, 0, 0)),
    "walls": dict(is_periodic=(0, 1, 0), bc_lo=(2, 0, 4), bc_hi=(2, 0, 5)),
    "sym": dict(is_periodic=(0, 0, 0), bc_lo=(3, 5, 1), bc_hi=(4, 2, 3)),
}


def padded_reference(state, geom, ng):
    """The domain grown by ng, every ghost from its source cell: separable
    per direction, so one np.pad per direction and per component."""
    out = state
    for d in range(3):
        ax = 3 - d  # (n, z, y, x)
        width = [(0, 0)] * 4
        width[ax] = (ng, ng)
        if geom.is_periodic[d]:
            out = np.pad(out, width, mode="wrap")
            continue
        parts = []
        for comp in range(10):
            c = out[comp:comp + 1]
            lo_w = [(0, 0)] * 4
            lo_w[ax] = (ng, 0)
            hi_w = [(0, 0)] * 4
            hi_w[ax] = (0, ng)
            res = c
            for side, word, w in ((0, geom.bc_lo[d], lo_w), (1, geom.bc_hi[d], hi_w)):
                mirror = word >= 3
                res = np.pad(res, w, mode="symmetric" if mirror else "edge")
                odd = (mirror and comp in (1, 2, 3) and
                       ((comp - 1 == d) or word == 5))
                if odd:
                    sl = [slice(None)] * 4
                    sl[ax] = slice(0, ng) if side == 0 else slice(-ng, None)
                    res[tuple(sl)] *= -1.0
            parts.append(res)
        out = np.concatenate(parts, axis=0)
    return out


def test_sfc_partition_balances_cells():
    boxes = hydro.level_boxes((64, 64, 32), (16, 16, 16))
    owner = D.sfc_partition(boxes, 4)
    cells = np.zeros(4)
    for (lo, hi), r in zip(boxes, owner):
        cells[r] += np.prod([hi[d] - lo[d] + 1 for d in range(3)])
    assert set(owner) == {0, 1, 2, 3}
    assert cells.max() / cells.min() <= 1.01
    # contiguous runs along the curve
    order = sorted(range(len(boxes)), key=lambda b: D.morton_key(boxes[b][0]))
    runs = [owner[b] for b in order]
    assert runs == sorted(runs)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, bcs, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n = (12, 10, 8)
        geom = hydro.make_geom(n, **BCSETS[bcs])
        boxes = hydro.level_boxes(n, (4, 5, 4))
        owner = D.sfc_partition(boxes, world)
        plan = D.GhostPlan(geom, boxes, 4)
        ex = D.Exchange(plan, owner, rank, world, torch.device("cpu"), dist)
        rng = np.random.default_rng(3)
        state = rng.standard_normal((10,) + tuple(n[::-1]))
        ref = padded_reference(state, geom, 4)
        src, dst = {}, {}
        for b, (lo, hi) in enumerate(boxes):
            if owner[b] != rank:
                continue
            src[b] = torch.from_numpy(np.ascontiguousarray(
                state[:, lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1]))
            t = torch.full((10, hi[2] - lo[2] + 9, hi[1] - lo[1] + 9, hi[0] - lo[0] + 9),
                           float("nan"), dtype=torch.float64)
            t[:, 4:-4, 4:-4, 4:-4] = src[b]
            dst[b] = t
        ex.fill(src, dst, "all", src_ng=0)
        bad = 0
        for b, t in dst.items():
            lo, hi = boxes[b]
            want = ref[:, lo[2]:hi[2] + 9, lo[1]:hi[1] + 9, lo[0]:hi[0] + 9]
            got = t.numpy()
            bad += int((got != want).sum())
        # the time-step minimum over the ranks
        est = torch.tensor([1.0 + rank], dtype=torch.float64)
        dist.all_reduce(est, op=dist.ReduceOp.MIN)
        q.put((rank, bad, len(dst), float(est.item())))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("bcs", list(BCSETS))
def test_ghost_exchange_two_ranks_matches_whole_domain_fill(bcs):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, bcs, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sum(r[2] for r in res) == len(hydro.level_boxes((12, 10, 8), (4, 5, 4)))
    for rank, bad, nbox, est in res:
        assert bad == 0, (rank, bad)
        assert nbox > 0
        assert est == 1.0
