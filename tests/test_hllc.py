"""The HLLC option (riemann_solver = 1).  The reference has no such solver,
so the only oracle is this project's CPU restatement (oracle/hydro_restate.cpp)
plus the exact solution of the Sod problem:

* the exact Riemann solver reproduces Toro's published Sod star state;
* Sod (x outflow, periodic y/z) with CTU-PLM and MOL-PLM: HLLC's density
  error against the exact solution is as small as riemannus's, and both
  converge;
* on the GPU, levels with HLLC match the restatement bit for bit (CTU-PPM
  blobs, MOL-PLM), and HLLC is rejected where it is not provided (EB).
"""
import numpy as np
import pytest

import oracle
from camr_b200 import problems as P

import exact_riemann as XR


def test_exact_riemann_sod_star_state():
    p, u = XR.star_state(1.0, 0.0, 1.0, 0.125, 0.0, 0.1)
    assert abs(p - 0.30313) < 1e-5 and abs(u - 0.92745) < 1e-5


def sod_run(nx, riemann, do_mol, t_end=0.15):
    n = (nx, 4, 4)
    dx = 1.0 / nx
    s = P.sod(n, (dx, dx, dx))
    p = oracle.default_params(do_mol=do_mol, ppm_type=0, cfl=0.3 if do_mol else 0.8,
                              riemann_solver=riemann)
    lev = oracle.make_level(n, periodic=(0, 1, 1), bc_lo=(2, 0, 0), bc_hi=(2, 0, 0),
                            dx=(dx, dx, dx))
    oracle.init_finalize("restate", p, lev, s)
    t, first, dtp = 0.0, True, 0.0
    while t < t_end - 1e-12:
        est = oracle.est_dt("restate", p, lev, s)
        dtp = min(est if first else min(est, 1.1 * dtp), t_end - t)
        oracle.advance_fixed_dt("restate", p, lev, s, [dtp])
        t += dtp
        first = False
    x = (np.arange(nx) + 0.5) * dx
    ex = XR.sample(x, t, 0.5, 1.0, 0.0, 1.0, 0.125, 0.0, 0.1)
    rho = s[P.URHO][2, 2, :]
    return np.abs(rho - ex[0]).mean()


@pytest.mark.parametrize("do_mol", [0, 1])
def test_hllc_sod_against_exact(do_mol):
    e_r = [sod_run(nx, 0, do_mol) for nx in (64, 128)]
    e_h = [sod_run(nx, 1, do_mol) for nx in (64, 128)]
    for e in (e_r, e_h):
        assert e[1] < 0.75 * e[0], e  # converging
    assert e_h[1] < 0.02 and e_h[1] < 1.3 * e_r[1], (e_h, e_r)


def acoustic_wave(n, amp=1e-3):
    """A small right-going acoustic wave along x (smooth, periodic)."""
    x = (np.arange(n[0]) + 0.5) / n[0]
    dr = amp * np.sin(2 * np.pi * x)[None, None, :] * np.ones((n[2], n[1], 1))
    g = 1.4
    rho = 1.0 + dr
    p = 1.0 + g * dr  # c = sqrt(1.4), p' = c^2 rho'
    u = np.sqrt(g) * dr
    s = np.zeros((P.NVAR, n[2], n[1], n[0]))
    s[P.URHO] = rho
    s[P.UMX] = rho * u
    s[P.UEINT] = p / (g - 1.0)
    s[P.UEDEN] = s[P.UEINT] + 0.5 * rho * u * u
    s[P.UFS] = rho
    return s


@pytest.mark.parametrize("case", ["shocky", "acoustic"])
def test_hllc_differs_from_riemannus_and_conserves(case):
    """Both solvers conserve mass on a periodic domain; on strong jumps they
    differ, on a small smooth wave they agree to the wave's second order."""
    n = (16, 16, 16) if case == "shocky" else (64, 4, 4)
    s = P.random_smooth(n, seed=9, amp=0.2, vel=0.3) if case == "shocky" else acoustic_wave(n)
    res = []
    for rs in (0, 1):
        p = oracle.default_params(do_mol=0, ppm_type=1, cfl=0.5, riemann_solver=rs)
        lev = oracle.make_level(n)
        a = s.copy()
        oracle.init_finalize("restate", p, lev, a)
        m0 = a[P.URHO].sum()
        oracle.advance("restate", p, lev, a, 10)
        assert abs(a[P.URHO].sum() - m0) <= 1e-12 * m0
        res.append(a)
    diff = np.abs(res[0][P.URHO] - res[1][P.URHO]).max()
    assert diff > 0.0
    if case == "acoustic":
        assert diff < 1e-5, diff


@pytest.mark.gpu
@pytest.mark.parametrize("do_mol,ppm", [(0, 1), (0, 0), (1, 0)])
def test_gpu_hllc_level_matches_restatement(do_mol, ppm):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from camr_b200 import hydro, native
    n = (32, 32, 32)
    s = P.blobs(n, tuple(1.0 / v for v in n), nblobs=4, seed=3)
    cfl = 0.3 if do_mol else 0.7
    p = oracle.default_params(do_mol=do_mol, ppm_type=ppm, cfl=cfl, riemann_solver=1)
    lev = oracle.make_level(n, max_grid_size=(16, 16, 16))
    ref = s.copy()
    oracle.init_finalize("restate", p, lev, ref)
    oracle.advance("restate", p, lev, ref, 4)
    prm = native.default_params(do_mol=do_mol, ppm_type=ppm, cfl=cfl, riemann_solver=1)
    L = hydro.Level(hydro.make_geom(n), prm, max_grid_size=(16, 16, 16))
    L.set_state(s)
    L.init_finalize()
    L.advance(4)
    got = L.get_state()
    assert np.array_equal(got, ref), np.abs(got - ref).max()
    L.close()


def test_hllc_rejected_where_not_provided(native_lib):
    """EB levels and the adjoint keep the reference solver only; the check
    happens before any CUDA call."""
    import ctypes as C

    from camr_b200 import hydro, native
    n = (8, 8, 8)
    geom = hydro.make_geom(n)
    prm = native.default_params(do_mol=1, cfl=0.3, riemann_solver=1)
    desc = native.LevelDesc()
    desc.geom = geom
    eb = native.EBGeom()
    h = C.c_void_p()
    st = native_lib.camr_eb_level_create(C.byref(desc), C.byref(eb), C.byref(prm), 1, None,
                                         C.byref(h))
    assert native.STATUS[st] == "CAMR_ERR_UNSUPPORTED"
    st = native_lib.camr_adjoint_create(C.byref(geom), C.byref(prm), 10, None, C.byref(h))
    assert native.STATUS[st] == "CAMR_ERR_UNSUPPORTED"
