"""Finite-difference checks of the adjoint's pointwise VJPs (CPU, no GPU).

The pointwise forward/VJP functions of camr_b200/csrc/adjoint_point.cuh
(face flux with edge states + two-shock Riemann + adjust_fluxes, MOL slopes
with the MC limiter, ctoprim, clean_state) are compiled for the host and
each VJP is compared with a central difference of its forward along random
directions: <b, (F(x+hv) - F(x-hv))/2h> against <J^T b, v>.  Samples that
straddle a kink (a limiter or Riemann branch switching inside [x-hv, x+hv])
may disagree; the test asks for agreement on nearly all samples.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "adjoint", "point_shim.cpp")
OUT = os.path.join(HERE, "adjoint", "_build", "libadj_point.so")

GAMMA = 1.4
PAR = np.array([GAMMA, 1e-8, 1e-7, 1e-200, 1e-12, 1e-8, 0.1, 1.0, 1e-4, 1e2, 0.0, 0.0])


@pytest.fixture(scope="module")
def lib():
    cxx = shutil.which("g++") or "/usr/bin/g++"
    deps = [SRC, os.path.join(HERE, "..", "camr_b200", "csrc", "adjoint_point.cuh")]
    if not os.path.exists(OUT) or any(os.path.getmtime(d) > os.path.getmtime(OUT) for d in deps):
        os.makedirs(os.path.dirname(OUT), exist_ok=True)
        subprocess.run([cxx, "-O2", "-ffp-contract=off", "-shared", "-fPIC", "-std=c++17", SRC,
                        "-o", OUT], check=True)
    L = C.CDLL(OUT)
    dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
    for name in ("adj_face_fwd", "adj_slope_fwd"):
        getattr(L, name).argtypes = [C.c_int, dp, dp, dp]
    for name in ("adj_face_vjp", "adj_slope_vjp"):
        getattr(L, name).argtypes = [C.c_int, dp, dp, dp, dp]
    for name in ("adj_ctoprim_fwd", "adj_clean_fwd"):
        getattr(L, name).argtypes = [dp, dp, dp]
    for name in ("adj_ctoprim_vjp", "adj_clean_vjp"):
        getattr(L, name).argtypes = [dp, dp, dp, dp]
    return L


def prim(rng, consistent=True):
    """A primitive record.  With a gamma-law EOS the internal-energy slope's
    left and right differences cancel to round-off (rho e = p/(gamma-1)), which
    puts that limiter exactly at its kink; `consistent=False` detunes rho e so
    that the slope VJP is tested off the kink."""
    rho = rng.uniform(0.3, 2.0)
    u = rng.uniform(-0.8, 0.8, size=3)
    p = rng.uniform(0.2, 5.0)
    y = rng.dirichlet([2.0, 2.0, 2.0])
    c = np.sqrt(GAMMA * p / rho)
    re = p / (GAMMA - 1.0) * (1.0 if consistent else rng.uniform(0.7, 1.3))
    return np.array([rho, u[0], u[1], u[2], p, re, y[0], y[1], y[2], c,
                     max(1e-8, 1e-8 * c)])


def cons(rng):
    q = prim(rng)
    rho, u = q[0], q[1:4]
    eint = q[5]
    U = np.zeros(10)
    U[0] = rho
    U[1:4] = rho * u
    U[5] = eint
    U[4] = eint + 0.5 * rho * (u @ u)
    U[6] = 300.0
    U[7:10] = rho * q[6:9]
    return U


def fd_check(fwd, vjp, x, nout, rng, h_rel=1e-7, nvec=3):
    errs = []
    for _ in range(nvec):
        v = rng.standard_normal(x.size) * (np.abs(x) + 1e-3)
        b = rng.standard_normal(nout)
        h = h_rel
        yp, ym = np.zeros(nout), np.zeros(nout)
        fwd(x + h * v, yp)
        fwd(x - h * v, ym)
        fd = b @ (yp - ym) / (2 * h)
        bx = np.zeros(x.size)
        vjp(x, b, bx)
        ad = bx @ v
        errs.append(abs(fd - ad) / max(abs(fd), abs(ad), 1e-12))
    return max(errs)


def summarize(errs):
    errs = np.array(errs)
    return np.median(errs), np.mean(errs < 1e-5)


@pytest.mark.parametrize("d", [0, 1, 2])
def test_face_vjp_matches_fd(lib, d):
    rng = np.random.default_rng(10 + d)
    par = PAR.copy()
    par[10] = 1.0 / 32     # dx
    par[11] = 1.0 / 32**2  # area
    errs = []
    for _ in range(300):
        qL, qR = prim(rng), prim(rng)
        sL = rng.standard_normal(8) * 0.05
        sR = rng.standard_normal(8) * 0.05
        dv = rng.uniform(-3.0, 1.0, size=4)
        x = np.concatenate([qL, qR, sL, sR, dv, cons(rng), cons(rng)])
        errs.append(fd_check(lambda a, y: lib.adj_face_fwd(d, par, a, y),
                             lambda a, b, bx: lib.adj_face_vjp(d, par, a, b, bx), x, 12, rng))
    med, ok = summarize(errs)
    assert med < 1e-7, med
    assert ok > 0.97, ok


@pytest.mark.parametrize("d", [0, 1, 2])
def test_slope_vjp_matches_fd(lib, d):
    rng = np.random.default_rng(20 + d)
    errs = []
    for _ in range(300):
        x = np.concatenate([prim(rng, False), prim(rng, False), prim(rng, False)])
        errs.append(fd_check(lambda a, y: lib.adj_slope_fwd(d, PAR, a, y),
                             lambda a, b, bx: lib.adj_slope_vjp(d, PAR, a, b, bx), x, 8, rng))
    med, ok = summarize(errs)
    assert med < 1e-7, med
    assert ok > 0.97, ok


def test_ctoprim_vjp_matches_fd(lib):
    rng = np.random.default_rng(30)
    errs = []
    for _ in range(300):
        x = cons(rng)
        errs.append(fd_check(lambda a, y: lib.adj_ctoprim_fwd(PAR, a, y),
                             lambda a, b, bx: lib.adj_ctoprim_vjp(PAR, a, b, bx), x, 11, rng))
    med, ok = summarize(errs)
    assert med < 1e-7 and ok > 0.99, (med, ok)


def test_clean_vjp_matches_fd(lib):
    rng = np.random.default_rng(40)
    errs = []
    for _ in range(300):
        x = cons(rng)
        # perturb energies off consistency so both reset branches are taken
        x[5] *= rng.uniform(0.9, 1.1)
        x[7:10] *= rng.uniform(0.95, 1.05, size=3)

        def fwd(a, y):
            lib.adj_clean_fwd(PAR, a, y)
            y[6] = 0.0  # UTEMP feeds nothing downstream

        def vjp(a, b, bx):
            b = b.copy()
            b[6] = 0.0
            lib.adj_clean_vjp(PAR, a, b, bx)

        errs.append(fd_check(fwd, vjp, x, 10, rng))
    med, ok = summarize(errs)
    assert med < 1e-7 and ok > 0.99, (med, ok)
