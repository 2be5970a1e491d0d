"""Failure of a rank in the cross-rank exchanges, on CPU (gloo): one rank
raises before the flux register's reflux and leaves; the other rank's
exchange must end with an error instead of waiting for good.  The failure is
made on the host; nothing here runs on a GPU."""
import os
import socket
import time
from datetime import timedelta

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from camr_b200 import distributed as D
from camr_b200 import hydro

N = (16, 12, 8)
MGS = (8, 6, 4)
FBOXES = [((2, 2, 2), (9, 9, 7)), ((10, 2, 2), (15, 7, 5)), ((28, 0, 12), (31, 5, 15))]
FOWNER = [0, 1, 1]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=10))
    try:
        rng = np.random.default_rng(rank)
        geom = hydro.make_geom(N)
        cboxes = hydro.level_boxes(N, MGS)
        cowner = D.sfc_partition(cboxes, world)
        fr = D.FluxRegister(geom, cboxes, cowner, FBOXES, FOWNER, rank, world,
                            torch.device("cpu"), dist)

        def faces(lo, hi, d):
            shape = [hi[e] - lo[e] + 1 + (e == d) for e in range(3)]
            return torch.from_numpy(rng.standard_normal((10,) + tuple(shape[::-1])))

        fr.crse_add({c: [faces(*cboxes[c], d) for d in range(3)] for c in fr.mine_c}, 0.5)
        fr.fine_add({b: [faces(*FBOXES[b], d) for d in range(3)] for b in fr.mine_f}, 0.25)
        if rank == 1:
            raise RuntimeError("injected failure before reflux")
        S = {c: torch.zeros((10,) + tuple(cboxes[c][1][e] - cboxes[c][0][e] + 1
                                          for e in (2, 1, 0)), dtype=torch.float64)
             for c in fr.mine_c}
        t0 = time.time()
        try:
            fr.reflux(S)
            q.put((rank, "completed", time.time() - t0))
        except Exception as exc:  # the survivor's exchange ends with an error
            q.put((rank, f"error: {type(exc).__name__}", time.time() - t0))
    except RuntimeError as exc:
        q.put((rank, f"injected: {exc}", 0.0))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def test_a_rank_that_leaves_ends_the_others_exchange_with_an_error():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        res = dict((r, (what, secs)) for r, what, secs in (q.get(timeout=120)
                                                           for _ in range(world)))
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert res[1][0].startswith("injected")
    assert res[0][0].startswith("error"), res[0]
    assert res[0][1] < 60.0
