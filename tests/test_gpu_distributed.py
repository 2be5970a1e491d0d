"""The box-distributed level driver (camr_b200/distributed.py) on one GPU:
with every box on the one rank, its steps -- the fab-level clean_state
parts, the planned ghost fills, camr_hydro_umdrv per box, the Saxpys and
the dt logic -- must reproduce the oracle's level steps over the same box
decomposition bit for bit.  (Several ranks need several GPUs; the exchange
between ranks is tested on CPU with gloo in tests/test_distributed.py.)"""
import numpy as np
import pytest

import oracle
from camr_b200 import distributed as D
from camr_b200 import hydro, native
from camr_b200 import problems as P

pytestmark = pytest.mark.gpu


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.parametrize("cfg,bcs", [
    (dict(do_mol=0, ppm_type=1, cfl=0.6), dict(periodic=(1, 1, 1), bc_lo=(0, 0, 0), bc_hi=(0, 0, 0))),
    (dict(do_mol=1, cfl=0.3), dict(periodic=(0, 1, 0), bc_lo=(2, 0, 4), bc_hi=(2, 0, 5))),
    (dict(do_mol=0, ppm_type=0, cfl=0.6, const_grav=-1.5),
     dict(periodic=(1, 1, 0), bc_lo=(0, 0, 4), bc_hi=(0, 0, 3))),
], ids=["ctu_ppm_periodic", "mol_walls", "ctu_plm_gravity"])
def test_distributed_level_one_rank_matches_oracle(cfg, bcs, oracle_kind, native_lib):
    torch = _torch()
    n = (24, 16, 16)
    mgs = (8, 8, 8)
    s0 = P.random_smooth(n, seed=19)
    p = oracle.default_params(**cfg)
    lev = oracle.make_level(n, max_grid_size=mgs, **bcs)
    ref = s0.copy()
    oracle.init_finalize(oracle_kind, p, lev, ref)
    start = ref.copy()
    _, hist, nass = oracle.advance(oracle_kind, p, lev, ref, 5)
    assert nass == 0
    geom = hydro.make_geom(n, is_periodic=bcs["periodic"], bc_lo=bcs["bc_lo"], bc_hi=bcs["bc_hi"])
    L = D.DistributedLevel(geom, native.default_params(**cfg), mgs, device=torch.device("cuda:0"))
    L.set_state(start)
    L.advance(5)
    got = L.get_state()
    assert hydro.get_error()[0] == 0
    assert L.dt_prev == hist[-1]
    nd = int((got != ref).sum())
    assert nd == 0, f"{nd} values differ"


class _Recorder:
    """Stands in for a flux register: keeps each call's fluxes and scale."""

    def __init__(self):
        self.calls = []

    def crse_add(self, fluxes, dtdx):
        self.calls.append(({b: [f.cpu().numpy().copy() for f in fl] for b, fl in fluxes.items()},
                           dtdx))


@pytest.mark.parametrize("cfg", [dict(do_mol=0, ppm_type=1, cfl=0.6), dict(do_mol=1, cfl=0.3)],
                         ids=["ctu_ppm", "mol"])
def test_distributed_level_feeds_flux_register(cfg, oracle_kind, native_lib):
    """The coarse level's hydro fluxes reach an attached flux register with
    construct_hydro_source's scale (one CrseAdd per CTU step, one per MOL
    stage at half weight), and the register's reflux of the level's new
    state equals the oracle's register given the same fluxes."""
    torch = _torch()
    n = (24, 16, 16)
    mgs = (8, 8, 8)
    fboxes = [((8, 8, 8), (23, 15, 15)), ((24, 8, 8), (31, 23, 15)),
              ((40, 0, 24), (47, 7, 31))]
    s0 = P.random_smooth(n, seed=23)
    p = oracle.default_params(**cfg)
    lev = oracle.make_level(n, max_grid_size=mgs)
    start = s0.copy()
    oracle.init_finalize(oracle_kind, p, lev, start)
    geom = hydro.make_geom(n)
    L = D.DistributedLevel(geom, native.default_params(**cfg), mgs, device=torch.device("cuda:0"))
    fr = D.FluxRegister(geom, L.boxes, L.owner, fboxes, [0] * len(fboxes),
                        device=torch.device("cuda:0"))
    rec = _Recorder()
    L.attach_flux_register(fr, "coarse")
    L.attach_flux_register(rec, "coarse")
    L.set_state(start)
    L.advance(1)
    assert hydro.get_error()[0] == 0
    dt = L.dt_prev
    vol = geom.dx[0] * geom.dx[1] * geom.dx[2]
    mol = cfg["do_mol"] == 1
    assert len(rec.calls) == (2 if mol else 1)
    for _, s in rec.calls:
        assert s == ((0.5 if mol else 1.0) * dt) / vol
    after = L.get_state()
    fr.reflux(L.S)
    got = L.get_state()
    want = np.ascontiguousarray(after.copy())
    cb = np.array([list(lo) + list(hi) for lo, hi in L.boxes])
    fb = np.array([list(lo) + list(hi) for lo, hi in fboxes])
    cfl = []
    for fl, _ in rec.calls:
        assert sorted(fl) == list(range(len(L.boxes)))
        cfl.append([fl[b] for b in range(len(L.boxes))])
    oracle.fluxreg_reflux("restate", lev, cb, cfl, rec.calls[0][1], fb, [], 0.0, want)
    nd = int((got.view(np.int64) != want.view(np.int64)).sum())
    assert nd == 0, f"{nd} values differ"
    assert (got != after).any()
