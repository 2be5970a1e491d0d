"""CPU tests of the oracle (no GPU).

* the restatement (oracle/hydro_restate.cpp) equals the reference's own
  per-box hydro compiled against the AMReX stand-in, bit for bit, for every
  method and boundary kind (skipped when oracle/_ref was not built);
* a single-level step is independent of the box / tile decomposition;
* physics sanity of the restated driver: exact Sod solution, conservation.
"""
import os

import numpy as np
import pytest

import oracle
from camr_b200 import problems as P

HAVE_REF = os.path.exists(oracle.lib_path("ref"))

CONFIGS = {
    "ctu_ppm": dict(do_mol=0, ppm_type=1),
    "ctu_plm": dict(do_mol=0, ppm_type=0),
    "ctu_plm_o2": dict(do_mol=0, ppm_type=0, plm_iorder=2),
    "ctu_ppm_noflat": dict(do_mol=0, ppm_type=1, use_flattening=0),
    "mol_plm": dict(do_mol=1, cfl=0.3),
}
BCSETS = {
    "periodic": dict(periodic=(1, 1, 1), bc_lo=(0, 0, 0), bc_hi=(0, 0, 0)),
    "walls": dict(periodic=(0, 1, 0), bc_lo=(2, 0, 4), bc_hi=(2, 0, 5)),
    "sym": dict(periodic=(0, 0, 0), bc_lo=(3, 5, 2), bc_hi=(4, 2, 3)),
    "inflow": dict(periodic=(0, 1, 0), bc_lo=(1, 0, 4), bc_hi=(2, 0, 1)),
}


def same_bits(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return int((~((a == b) | (np.isnan(a) & np.isnan(b)))).sum())


@pytest.fixture(scope="module", autouse=True)
def _built():
    if not os.path.exists(oracle.lib_path("restate")):
        oracle.build(ref=False)


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built (reference sources absent)")
@pytest.mark.parametrize("cfg", list(CONFIGS))
@pytest.mark.parametrize("bcs", list(BCSETS))
def test_restatement_equals_reference_box(cfg, bcs):
    n = (11, 9, 8)
    lev = oracle.make_level(n, **BCSETS[bcs])
    p = oracle.default_params(**CONFIGS[cfg])
    s = P.random_smooth(n, seed=2)
    oracle.init_finalize("ref", p, lev, s)
    border = oracle.expand_state("ref", p, lev, s)
    assert same_bits(border, oracle.expand_state("restate", p, lev, s)) == 0
    dt = 0.5 * oracle.est_dt("ref", p, lev, s)
    lo, hi = [0, 0, 0], [n[0] - 1, n[1] - 1, n[2] - 1]
    args = (p, lo, hi, lo, hi, list(lev.bc_lo), list(lev.bc_hi), border, [-4, -4, -4],
            list(lev.dx), dt)
    a = oracle.hydro_box("restate", *args)
    b = oracle.hydro_box("ref", *args)
    assert a[2] == 0 and b[2] == 0
    assert same_bits(a[0], b[0]) == 0
    for d in range(3):
        assert same_bits(a[1][d], b[1][d]) == 0


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built (reference sources absent)")
@pytest.mark.parametrize("cfg", list(CONFIGS))
def test_restatement_equals_reference_subbox(cfg):
    """A box inside a larger domain whose index space starts at (-3, 2, 0),
    touching only the z-low wall."""
    n = (20, 16, 12)
    dlo = (-3, 2, 0)
    lev = oracle.make_level(n, lo=dlo, periodic=(0, 1, 0), bc_lo=(1, 0, 4), bc_hi=(2, 0, 5))
    p = oracle.default_params(**CONFIGS[cfg])
    s = P.random_smooth(n, seed=8)
    oracle.init_finalize("ref", p, lev, s)
    border = oracle.expand_state("ref", p, lev, s)
    assert same_bits(border, oracle.expand_state("restate", p, lev, s)) == 0
    dt = 0.5 * oracle.est_dt("ref", p, lev, s)
    lo, hi = [2, 5, 0], [11, 12, 6]
    dhi = [dlo[d] + n[d] - 1 for d in range(3)]
    args = (p, lo, hi, list(dlo), dhi, list(lev.bc_lo), list(lev.bc_hi), border,
            [dlo[d] - 4 for d in range(3)], list(lev.dx), dt)
    a = oracle.hydro_box("restate", *args)
    b = oracle.hydro_box("ref", *args)
    assert a[2] == 0 and b[2] == 0
    assert same_bits(a[0], b[0]) == 0
    for d in range(3):
        assert same_bits(a[1][d], b[1][d]) == 0


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built (reference sources absent)")
@pytest.mark.parametrize("cfg", ["ctu_ppm", "mol_plm"])
def test_restatement_equals_reference_run(cfg):
    n = (16, 12, 10)
    bcs = BCSETS["walls"]
    p = oracle.default_params(**CONFIGS[cfg])
    out = {}
    for kind in ("ref", "restate"):
        lev = oracle.make_level(n, **bcs)
        s = P.random_smooth(n, seed=9)
        oracle.init_finalize(kind, p, lev, s)
        _, hist, nass = oracle.advance(kind, p, lev, s, 3)
        assert nass == 0
        out[kind] = (s, hist)
    assert same_bits(out["ref"][0], out["restate"][0]) == 0
    assert same_bits(out["ref"][1], out["restate"][1]) == 0


@pytest.mark.parametrize("cfg", ["ctu_ppm", "ctu_plm", "mol_plm"])
def test_decomposition_independence(cfg):
    """The reference's per-tile hydro gives the same bits for any tiling."""
    kind = "ref" if HAVE_REF else "restate"
    n = (20, 12, 12)
    p = oracle.default_params(**CONFIGS[cfg])
    res = []
    for ts, mgs in [((0, 0, 0), (0, 0, 0)), ((8, 4, 4), (0, 0, 0)), ((5, 3, 7), (10, 12, 6))]:
        lev = oracle.make_level(n, tile_size=ts, max_grid_size=mgs, **BCSETS["walls"])
        s = P.random_smooth(n, seed=4)
        oracle.init_finalize(kind, p, lev, s)
        oracle.advance(kind, p, lev, s, 2)
        res.append(s)
    assert same_bits(res[0], res[1]) == 0
    assert same_bits(res[0], res[2]) == 0


def exact_sod_density(x, t, gamma=1.4, rl=1.0, pl=1.0, rr=0.125, pr=0.1, x0=0.5):
    """Density of the exact Sod solution (Toro, ch. 4), zero initial velocities."""
    cl = np.sqrt(gamma * pl / rl)
    cr = np.sqrt(gamma * pr / rr)

    def f(p, rk, pk, ck):
        if p > pk:
            a = 2.0 / ((gamma + 1) * rk)
            b = (gamma - 1) / (gamma + 1) * pk
            return (p - pk) * np.sqrt(a / (p + b))
        return 2 * ck / (gamma - 1) * ((p / pk) ** ((gamma - 1) / (2 * gamma)) - 1)

    lo, hi = 1e-8, 10.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if f(mid, rl, pl, cl) + f(mid, rr, pr, cr) > 0:
            hi = mid
        else:
            lo = mid
    ps = 0.5 * (lo + hi)
    us = 0.5 * (f(ps, rr, pr, cr) - f(ps, rl, pl, cl))
    rsl = rl * (ps / pl) ** (1 / gamma)
    rsr = rr * ((ps / pr + (gamma - 1) / (gamma + 1)) / ((gamma - 1) / (gamma + 1) * ps / pr + 1))
    s_shock = us * rsr / (rsr - rr) if rsr != rr else us
    s_shock = np.sqrt(gamma * pr / rr) * np.sqrt((gamma + 1) / (2 * gamma) * ps / pr +
                                                 (gamma - 1) / (2 * gamma))
    csl = cl * (ps / pl) ** ((gamma - 1) / (2 * gamma))
    out = np.empty_like(x)
    for n, xv in enumerate(x):
        s = (xv - x0) / t
        if s < -cl:
            out[n] = rl
        elif s < us - csl:
            u = 2 / (gamma + 1) * (cl + s)
            c = cl - (gamma - 1) / 2 * u
            out[n] = rl * (c / cl) ** (2 / (gamma - 1))
        elif s < us:
            out[n] = rsl
        elif s < s_shock:
            out[n] = rsr
        else:
            out[n] = rr
    return out


@pytest.mark.parametrize("method", ["ctu_plm", "ctu_ppm", "mol_plm"])
def test_sod_against_exact_solution(method):
    """Physics check (not parity): 1-D Sod profile converges to the exact solution."""
    kind = "ref" if HAVE_REF else "restate"
    nx = 128
    n = (nx, 4, 4)
    dx = (1.0 / nx, 1.0 / nx, 1.0 / nx)
    cfg = dict(CONFIGS[method])
    p = oracle.default_params(**cfg)
    lev = oracle.make_level(n, dx=dx, periodic=(0, 1, 1), bc_lo=(2, 0, 0), bc_hi=(2, 0, 0))
    s = P.sod(n, dx)
    oracle.init_finalize(kind, p, lev, s)
    t = 0.0
    dt_prev = 0.0
    first = True
    while t < 0.15:
        dt_prev, hist, _ = oracle.advance(kind, p, lev, s, 1, first_step=first, dt_prev=dt_prev)
        first = False
        t += hist[0]
    x = (np.arange(nx) + 0.5) / nx
    rho = s[0, 2, 2, :]
    err = np.abs(rho - exact_sod_density(x, t)).mean()
    assert err < 0.01, err


@pytest.mark.parametrize("cfg", ["ctu_ppm", "mol_plm"])
def test_conservation_periodic_oracle(cfg):
    kind = "ref" if HAVE_REF else "restate"
    n = (16, 12, 10)
    p = oracle.default_params(**CONFIGS[cfg])
    lev = oracle.make_level(n, **BCSETS["periodic"])
    s = P.random_smooth(n, seed=8)
    oracle.init_finalize(kind, p, lev, s)
    a = s.copy()
    oracle.advance(kind, p, lev, s, 4)
    for comp in range(5):
        scale = np.abs(a[comp]).sum()
        assert abs(s[comp].sum() - a[comp].sum()) <= 1e-12 * scale


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built (reference sources absent)")
@pytest.mark.parametrize("cfg", ["ctu_ppm", "ctu_plm", "mol_plm"])
def test_reference_full_interface_equals_per_box_call(cfg):
    """The reference's hydro_umdrv driven with caller q/qaux/src_q from its own
    ctoprim/srctoprim and Cartesian area/volume arrays gives the same bits as
    the per-box glue that computes them (the pin of the full-interface
    oracle used by the GPU test of camr_hydro_umdrv_full)."""
    n = (10, 9, 8)
    lev = oracle.make_level(n, **BCSETS["walls"])
    p = oracle.default_params(**CONFIGS[cfg])
    s = P.random_smooth(n, seed=4)
    oracle.init_finalize("ref", p, lev, s)
    border = oracle.expand_state("ref", p, lev, s)
    rng = np.random.default_rng(2)
    src = rng.standard_normal(border.shape) * 0.2
    dt = 0.5 * oracle.est_dt("ref", p, lev, s)
    lo, hi = [0, 0, 0], [n[0] - 1, n[1] - 1, n[2] - 1]
    glo, ghi = [-4, -4, -4], [n[0] + 3, n[1] + 3, n[2] + 3]
    q, qaux, srcq = oracle.ref_ctoprim(p, glo, ghi, border, glo, src=src)
    dx = list(lev.dx)
    area = [np.full((n[2] + (d == 2), n[1] + (d == 1), n[0] + (d == 0)),
                    (dx[1] * dx[2], dx[0] * dx[2], dx[0] * dx[1])[d]) for d in range(3)]
    vol = np.full((n[2], n[1], n[0]), dx[0] * dx[1] * dx[2])
    d1, f1, nass = oracle.ref_hydro_box_full(p, lo, hi, lo, hi, list(lev.bc_lo), list(lev.bc_hi),
                                             border, glo, q, qaux, srcq, area, vol, dx, dt)
    assert nass == 0
    d0, f0, nass = oracle.hydro_box("ref", p, lo, hi, lo, hi, list(lev.bc_lo), list(lev.bc_hi),
                                    border, glo, dx, dt, src=src)
    assert nass == 0
    assert same_bits(d1, d0) == 0
    for d in range(3):
        assert same_bits(f1[d], f0[d]) == 0
