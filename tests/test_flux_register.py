"""The two-level flux register across ranks (camr_b200/distributed.py
FluxRegister) on CPU, against the oracle's restated YAFluxRegister
(oracle/level_driver.cpp make_fluxreg / crse_add / fine_add and the reflux
of post_timestep, through orc_fluxreg_reflux), bit for bit.

The fine boxes are placed so that the register meets its corner cases: two
fine boxes touching the same uncovered coarse cell from different sides
(its contributions must be added in the single-process box order), fine
boxes whose neighbours wrap around the periodic domain, a one-coarse-cell
fine box, fine boxes owned by one rank correcting coarse cells owned by the
other, and signed zeros in the state (the reflux adds +0 to every cell)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from camr_b200 import distributed as D
from camr_b200 import hydro, native

N = (16, 12, 8)
MGS = (8, 6, 4)
FBOXES = [((2, 2, 2), (9, 9, 7)),       # coarse 1..4 x 1..4 x 1..3
          ((10, 2, 2), (15, 7, 5)),     # touches the first along x
          ((28, 0, 12), (31, 5, 15)),   # neighbours across the periodic x, y and z edges
          ((20, 16, 4), (21, 17, 5)),   # one coarse cell
          ((0, 18, 0), (3, 23, 1))]     # low x and high y edges
NCALL = 4   # two subcycles of a two-stage fine step
DTDX_C, DTDX_F = 0.37, 0.1825


def _inputs():
    """Seeded coarse state, coarse face fluxes and fine face fluxes."""
    rng = np.random.default_rng(11)
    cboxes = hydro.level_boxes(N, MGS)
    S = rng.standard_normal((10,) + N[::-1])
    S[3, 0, 0, :4] = -0.0
    S[2, 1, 2, 5:9] = 0.0

    def faces(lo, hi, d):
        shape = [hi[e] - lo[e] + 1 + (e == d) for e in range(3)]
        f = rng.standard_normal((10,) + tuple(shape[::-1]))
        f[:, 0, 0, 0] = 0.0
        return f

    cflux = [[faces(lo, hi, d) for d in range(3)] for lo, hi in cboxes]
    fflux = [[[faces(lo, hi, d) for d in range(3)] for lo, hi in FBOXES]
             for _ in range(NCALL)]
    return cboxes, S, cflux, fflux


def _oracle(cboxes, S, cflux, fflux):
    import oracle
    lev = oracle.make_level(N)
    out = np.ascontiguousarray(S.copy())
    cb = np.array([list(lo) + list(hi) for lo, hi in cboxes])
    fb = np.array([list(lo) + list(hi) for lo, hi in FBOXES])
    oracle.fluxreg_reflux("restate", lev, cb, [cflux], DTDX_C, fb, fflux, DTDX_F, out)
    return out


def _run_rank(rank, world, cowner, fowner, pg, ng, device=None):
    device = device or torch.device("cpu")
    cboxes, S, cflux, fflux = _inputs()
    geom = hydro.make_geom(N)
    fr = D.FluxRegister(geom, cboxes, cowner, FBOXES, fowner, rank, world, device, pg)
    fr.crse_add({c: [torch.from_numpy(a).to(device) for a in cflux[c]] for c in fr.mine_c},
                DTDX_C)
    for call in range(NCALL):
        fr.fine_add({b: [torch.from_numpy(a).to(device) for a in fflux[call][b]]
                     for b in fr.mine_f}, DTDX_F)
    mine = {}
    for c in fr.mine_c:
        lo, hi = cboxes[c]
        part = S[:, lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1]
        t = torch.full((10,) + tuple(hi[e] - lo[e] + 1 + 2 * ng for e in (2, 1, 0)), np.nan,
                       dtype=torch.float64)
        t[:, ng:t.shape[1] - ng, ng:t.shape[2] - ng, ng:t.shape[3] - ng] = torch.from_numpy(part)
        mine[c] = t.to(device)
    fr.reflux(mine, ng)
    out = {}
    for c, t in mine.items():
        out[c] = t[:, ng:t.shape[1] - ng, ng:t.shape[2] - ng,
                   ng:t.shape[3] - ng].cpu().numpy().copy()
    return out, fr


def _assemble(cboxes, parts):
    full = np.full((10,) + N[::-1], np.nan)
    for c, a in parts.items():
        lo, hi = cboxes[c]
        full[:, lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1] = a
    return full


def _same_bits(a, b):
    return np.array_equal(a.view(np.int64), b.view(np.int64))


def test_flux_register_one_rank_matches_oracle(oracle_kind):
    cboxes, S, cflux, fflux = _inputs()
    want = _oracle(cboxes, S, cflux, fflux)
    assert not _same_bits(want, S)        # the register changed something
    parts, fr = _run_rank(0, 1, [0] * len(cboxes), [0] * len(FBOXES), None, 2)
    got = _assemble(cboxes, parts)
    assert _same_bits(got, want)
    # a cell that two fine boxes correct (coarse (5, 4, 1): x+ of the first
    # box, y+ of the second) takes more than one box side's 4 sub-faces per
    # fine call
    assert len(fr._rounds) > 4


@pytest.mark.gpu
def test_flux_register_on_device_matches_oracle(oracle_kind):
    """The same register with its tensors (register, plan indices, fluxes,
    states) in device memory: the products, sums and scatters then run as
    device kernels and must still give the oracle's bits."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    cboxes, S, cflux, fflux = _inputs()
    want = _oracle(cboxes, S, cflux, fflux)
    parts, fr = _run_rank(0, 1, [0] * len(cboxes), [0] * len(FBOXES), None, 1,
                          torch.device("cuda:0"))
    assert fr.d.is_cuda
    assert _same_bits(_assemble(cboxes, parts), want)


def test_flux_register_comparison_sees_the_order(oracle_kind):
    """The oracle given the fine boxes in reverse order (its additions to a
    cell that two boxes correct then come in the other order) differs from
    the register in some bits: the bit-for-bit comparisons above check the
    order of the additions, not only their sum."""
    import oracle
    cboxes, S, cflux, fflux = _inputs()
    rev = np.ascontiguousarray(S.copy())
    cb = np.array([list(lo) + list(hi) for lo, hi in cboxes])
    fb = np.array([list(lo) + list(hi) for lo, hi in FBOXES[::-1]])
    oracle.fluxreg_reflux("restate", oracle.make_level(N), cb, [cflux], DTDX_C, fb,
                          [call[::-1] for call in fflux], DTDX_F, rev)
    parts, _ = _run_rank(0, 1, [0] * len(cboxes), [0] * len(FBOXES), None, 0)
    got = _assemble(cboxes, parts)
    assert not _same_bits(got, rev)
    assert np.allclose(got, rev, rtol=0, atol=1e-12)


def test_flux_register_rejects_bad_boxes():
    geom = hydro.make_geom(N)
    cboxes = hydro.level_boxes(N, MGS)
    with pytest.raises(ValueError):
        D.FluxRegister(geom, cboxes, [0] * len(cboxes), [((1, 0, 0), (4, 3, 3))], [0])
    with pytest.raises(ValueError):
        D.FluxRegister(geom, cboxes, [0] * len(cboxes),
                       [((0, 0, 0), (3, 3, 3)), ((2, 2, 2), (5, 5, 5))], [0, 0])
    walls = hydro.make_geom(N, is_periodic=(0, 1, 1), bc_lo=(2, 0, 0), bc_hi=(2, 0, 0))
    with pytest.raises(ValueError):
        D.FluxRegister(walls, cboxes, [0] * len(cboxes), FBOXES, [0] * len(FBOXES))
    # every two-level piece refuses boxes outside the domain, overlapping
    # coarse boxes and coarse boxes that leave cells uncovered
    for cls in (D.FluxRegister, D.AverageDown, D.TwoLevelFill):
        with pytest.raises(ValueError, match="outside the domain"):
            cls(geom, cboxes, [0] * len(cboxes), [((30, 0, 0), (33, 3, 3))], [0])
        with pytest.raises(ValueError, match="outside the domain"):
            cls(geom, cboxes, [0] * len(cboxes), [((-4, 0, 0), (-1, 3, 3))], [0])
        with pytest.raises(ValueError, match="overlaps"):
            cls(geom, cboxes + [cboxes[0]], [0] * (len(cboxes) + 1), FBOXES, [0] * len(FBOXES))
        with pytest.raises(ValueError, match="do not cover"):
            cls(geom, cboxes[1:], [0] * (len(cboxes) - 1), FBOXES, [0] * len(FBOXES))
        with pytest.raises(ValueError, match="not aligned"):
            cls(geom, cboxes, [0] * len(cboxes), [((1, 0, 0), (4, 3, 3))], [0])


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, fowner, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cboxes = hydro.level_boxes(N, MGS)
        cowner = D.sfc_partition(cboxes, world)
        parts, fr = _run_rank(rank, world, cowner, fowner, dist, 1)
        q.put((rank, parts, len(fr._send), len(fr._recv_pos)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,fowner", [(2, [0, 1, 0, 1, 1]), (2, [1, 1, 1, 1, 1]),
                                          (3, [2, 0, 1, 2, 0])])
def test_flux_register_several_ranks_matches_oracle(oracle_kind, world, fowner):
    cboxes, S, cflux, fflux = _inputs()
    want = _oracle(cboxes, S, cflux, fflux)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, fowner, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    parts = {}
    for rank, pr, nsend, nrecv in res:
        assert not set(pr) & set(parts)
        parts.update(pr)
        if world == 2 and rank == 1:
            assert nsend == 2     # fine boxes of rank 1 correct cells of both ranks
    got = _assemble(cboxes, parts)
    assert _same_bits(got, want)


# ---- average-down across ranks (distributed.AverageDown) ----

def _fine_states():
    rng = np.random.default_rng(29)
    out = []
    for lo, hi in FBOXES:
        a = rng.standard_normal((10,) + tuple(hi[e] - lo[e] + 1 for e in (2, 1, 0)))
        a[1, 0, 0, :2] = -0.0
        out.append(a)
    return out


def _avg_oracle(S):
    import oracle
    out = np.ascontiguousarray(S.copy())
    fb = np.array([list(lo) + list(hi) for lo, hi in FBOXES])
    oracle.avg_down("restate", oracle.make_level(N), fb, _fine_states(), out)
    return out


def _avg_rank(rank, world, cowner, fowner, pg, ng, device=None):
    device = device or torch.device("cpu")
    cboxes, S, _, _ = _inputs()
    fs = _fine_states()
    ad = D.AverageDown(hydro.make_geom(N), cboxes, cowner, FBOXES, fowner, rank, world,
                       device, pg)
    fine = {}
    for b in ad.mine_f:
        t = torch.full((10,) + tuple(s + 2 * ng for s in fs[b].shape[1:]), np.nan,
                       dtype=torch.float64)
        t[:, ng:t.shape[1] - ng, ng:t.shape[2] - ng, ng:t.shape[3] - ng] = torch.from_numpy(fs[b])
        fine[b] = t.to(device)
    crse = {}
    for c, (lo, hi) in enumerate(cboxes):
        if cowner[c] != rank:
            continue
        t = torch.full((10,) + tuple(hi[e] - lo[e] + 1 + 2 * ng for e in (2, 1, 0)), np.nan,
                       dtype=torch.float64)
        t[:, ng:t.shape[1] - ng, ng:t.shape[2] - ng, ng:t.shape[3] - ng] = torch.from_numpy(
            S[:, lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1])
        crse[c] = t.to(device)
    ad(fine, crse, ng_f=ng, ng_c=ng)
    return {c: t[:, ng:t.shape[1] - ng, ng:t.shape[2] - ng,
                 ng:t.shape[3] - ng].cpu().numpy().copy() for c, t in crse.items()}


def test_average_down_one_rank_matches_oracle(oracle_kind):
    cboxes, S, _, _ = _inputs()
    want = _avg_oracle(S)
    assert not _same_bits(want, S)
    got = _assemble(cboxes, _avg_rank(0, 1, [0] * len(cboxes), [0] * len(FBOXES), None, 2))
    assert _same_bits(got, want)


@pytest.mark.gpu
def test_average_down_on_device_matches_oracle(oracle_kind):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    cboxes, S, _, _ = _inputs()
    want = _avg_oracle(S)
    got = _assemble(cboxes, _avg_rank(0, 1, [0] * len(cboxes), [0] * len(FBOXES), None, 1,
                                      torch.device("cuda:0")))
    assert _same_bits(got, want)


def _avg_worker(rank, world, port, fowner, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cboxes = hydro.level_boxes(N, MGS)
        q.put((rank, _avg_rank(rank, world, D.sfc_partition(cboxes, world), fowner, dist, 1)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,fowner", [(2, [0, 1, 0, 1, 1]), (2, [1, 1, 1, 1, 1]),
                                          (3, [2, 0, 1, 2, 0])])
def test_average_down_several_ranks_matches_oracle(oracle_kind, world, fowner):
    cboxes, S, _, _ = _inputs()
    want = _avg_oracle(S)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_avg_worker, args=(r, world, port, fowner, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    parts = {}
    for _, pr in res:
        assert not set(pr) & set(parts)
        parts.update(pr)
    assert _same_bits(_assemble(cboxes, parts), want)


def test_flux_register_two_coarse_calls_and_reset(oracle_kind):
    """Two CrseAdd calls per coarse step (the MOL stages) accumulate in call
    order as the oracle's register does; after reset() a reflux with no new
    calls leaves the state's values as they are (it adds +0)."""
    import oracle
    cboxes, S, cflux, fflux = _inputs()
    rng = np.random.default_rng(12)
    cflux2 = [[rng.standard_normal(a.shape) for a in per] for per in cflux]
    want = np.ascontiguousarray(S.copy())
    cb = np.array([list(lo) + list(hi) for lo, hi in cboxes])
    fb = np.array([list(lo) + list(hi) for lo, hi in FBOXES])
    oracle.fluxreg_reflux("restate", oracle.make_level(N), cb, [cflux, cflux2], DTDX_C, fb,
                          fflux, DTDX_F, want)
    fr = D.FluxRegister(hydro.make_geom(N), cboxes, [0] * len(cboxes), FBOXES,
                        [0] * len(FBOXES))
    for calls in (cflux, cflux2):
        fr.crse_add({c: [torch.from_numpy(a) for a in calls[c]] for c in fr.mine_c}, DTDX_C)
    for call in range(NCALL):
        fr.fine_add({b: [torch.from_numpy(a) for a in fflux[call][b]] for b in fr.mine_f},
                    DTDX_F)
    mine = {}
    for c, (lo, hi) in enumerate(cboxes):
        mine[c] = torch.from_numpy(np.ascontiguousarray(
            S[:, lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1]))
    fr.reflux(mine)
    got = _assemble(cboxes, {c: t.numpy() for c, t in mine.items()})
    assert _same_bits(got, want)
    fr.reset()
    fr.reflux(mine)
    again = _assemble(cboxes, {c: t.numpy() for c, t in mine.items()})
    assert np.array_equal(again, want)


def test_level_refuses_a_register_on_other_boxes(native_lib):
    """attach_flux_register checks that the register's boxes of that role are
    the level's own boxes (no device work: the level is only constructed)."""
    geom = hydro.make_geom(N)
    L = D.DistributedLevel(geom, native.default_params(), MGS, device=torch.device("cpu"))
    ok = D.FluxRegister(geom, L.boxes, L.owner, FBOXES, [0] * len(FBOXES))
    L.attach_flux_register(ok, "coarse")
    other = hydro.level_boxes(N, (4, 6, 4))
    bad = D.FluxRegister(geom, other, [0] * len(other), FBOXES, [0] * len(FBOXES))
    with pytest.raises(ValueError, match="coarse boxes"):
        L.attach_flux_register(bad, "coarse")
    with pytest.raises(ValueError, match="fine boxes"):
        L.attach_flux_register(ok, "fine")
    with pytest.raises(ValueError):
        L.attach_flux_register(ok, "middle")
