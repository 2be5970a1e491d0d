"""GPU test of the allocation-free per-box hydro (camr_hydro_umdrv_noalloc).

Callers that may not allocate device memory while they run (arena-owned
memory, real-time loops, plugin hosts) use this entry point; its scratch is a
fixed static device array.  This file is collected last on purpose.  Each
case calls the new entry point twice in a row (the scratch keeps the
previous call's contents) and compares both results with the existing
camr_hydro_umdrv through the C ABI, with the bit-exact tolerance the other
parity tests use; an oversized box must be rejected with CAMR_ERR_INVALID.
"""
import ctypes as C

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


def _call(lib_fn, lo, hi, geom, uin, dsdt, flx, prm, dt):
    from camr_b200 import hydro
    fu = hydro.fab_of(uin, [lo[d] - 4 for d in range(3)])
    fd = hydro.fab_of(dsdt, lo)
    ff = [hydro.fab_of(f, lo) for f in flx]
    return lib_fn(C.byref((C.c_int * 3)(*lo)), C.byref((C.c_int * 3)(*hi)), C.byref(geom),
                  C.byref(fu), None, C.byref(fd), C.byref(ff[0]), C.byref(ff[1]),
                  C.byref(ff[2]), C.byref(prm), float(dt), None)


def _fresh(torch, n, base):
    dev = torch.device("cuda:0")
    dsdt = torch.from_numpy(base.copy()).to(dev)
    flx = []
    for d in range(3):
        sh = list(n)
        sh[d] += 1
        flx.append(torch.full((10, sh[2], sh[1], sh[0]), float("nan"), dtype=torch.float64,
                              device=dev))
    return dsdt, flx


@pytest.mark.parametrize("case", [
    dict(n=(13, 10, 9), cfg=dict(do_mol=0, ppm_type=1), periodic=(1, 1, 1),
         bc_lo=(0, 0, 0), bc_hi=(0, 0, 0)),
    dict(n=(16, 12, 20), cfg=dict(do_mol=1, cfl=0.3), periodic=(0, 1, 0),
         bc_lo=(2, 0, 4), bc_hi=(2, 0, 5)),
])
def test_noalloc_matches_allocating_entry_point(case, native_lib):
    torch = _torch()
    from camr_b200 import hydro, native
    n = case["n"]
    lev = oracle.make_level(n, periodic=case["periodic"], bc_lo=case["bc_lo"],
                            bc_hi=case["bc_hi"])
    kind = "restate"
    if not __import__("os").path.exists(oracle.lib_path(kind)):
        oracle.build(ref=False)
    p_or = oracle.default_params(**case["cfg"])
    s = P.random_smooth(n, seed=21)
    oracle.init_finalize(kind, p_or, lev, s)
    border = oracle.expand_state(kind, p_or, lev, s)
    dt = 0.5 * oracle.est_dt(kind, p_or, lev, s)
    geom = hydro.make_geom(n, is_periodic=case["periodic"], bc_lo=case["bc_lo"],
                           bc_hi=case["bc_hi"])
    prm = native.default_params(**case["cfg"])
    uin = torch.from_numpy(border).to("cuda:0")
    lo = [0, 0, 0]
    hi = [n[0] - 1, n[1] - 1, n[2] - 1]
    base = np.full((10, n[2], n[1], n[0]), 0.5)

    d_ref, f_ref = _fresh(torch, n, base)
    assert _call(native_lib.camr_hydro_umdrv, lo, hi, geom, uin, d_ref, f_ref, prm, dt) == 0
    torch.cuda.synchronize()
    want = [d_ref.cpu().numpy()] + [f.cpu().numpy() for f in f_ref]

    for call in range(2):  # two calls in a row share the scratch
        d_new, f_new = _fresh(torch, n, base)
        st = _call(native_lib.camr_hydro_umdrv_noalloc, lo, hi, geom, uin, d_new, f_new, prm, dt)
        assert st == 0, native_lib.camr_noalloc_last_error()
        torch.cuda.synchronize()
        got = [d_new.cpu().numpy()] + [f.cpu().numpy() for f in f_new]
        for g, w, what in zip(got, want, ["dsdt", "flux x", "flux y", "flux z"]):
            same = (g == w) | (np.isnan(g) & np.isnan(w))
            assert same.all(), f"call {call}: {what}: {int((~same).sum())} values differ"


def test_noalloc_rejects_boxes_beyond_the_scratch(native_lib):
    torch = _torch()
    from camr_b200 import hydro, native
    n = (40, 40, 40)  # a CTU box this size needs more than the 64 MiB scratch
    geom = hydro.make_geom(n)
    prm = native.default_params(do_mol=0, ppm_type=1)
    uin = torch.ones((10, n[2] + 8, n[1] + 8, n[0] + 8), dtype=torch.float64, device="cuda:0")
    dsdt, flx = _fresh(torch, n, np.zeros((10, n[2], n[1], n[0])))
    st = _call(native_lib.camr_hydro_umdrv_noalloc, [0, 0, 0], [39, 39, 39], geom, uin, dsdt,
               flx, prm, 1e-3)
    assert native.STATUS[st] == "CAMR_ERR_INVALID"
    assert b"static scratch" in native_lib.camr_noalloc_last_error()


def test_noalloc_rejects_a_source_box_beyond_the_scratch(native_lib):
    """A 28^3 CTU box fits without a source fab but not with one."""
    torch = _torch()
    from camr_b200 import hydro, native
    n = (28, 28, 28)
    geom = hydro.make_geom(n)
    prm = native.default_params(do_mol=0, ppm_type=1)
    uin = torch.ones((10, n[2] + 8, n[1] + 8, n[0] + 8), dtype=torch.float64, device="cuda:0")
    src = torch.zeros_like(uin)
    dsdt, flx = _fresh(torch, n, np.zeros((10, n[2], n[1], n[0])))
    lo, hi = [0, 0, 0], [27, 27, 27]
    fu = hydro.fab_of(uin, [-4, -4, -4])
    fs = hydro.fab_of(src, [-4, -4, -4])
    fd = hydro.fab_of(dsdt, lo)
    ff = [hydro.fab_of(f, lo) for f in flx]
    st = native_lib.camr_hydro_umdrv_noalloc(
        C.byref((C.c_int * 3)(*lo)), C.byref((C.c_int * 3)(*hi)), C.byref(geom), C.byref(fu),
        C.byref(fs), C.byref(fd), C.byref(ff[0]), C.byref(ff[1]), C.byref(ff[2]),
        C.byref(prm), 1e-3, None)
    assert native.STATUS[st] == "CAMR_ERR_INVALID"
    assert b"static scratch" in native_lib.camr_noalloc_last_error()
