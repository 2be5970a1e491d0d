"""CPU checks of the C ABI: the library loads and exports every entry point
include/camr_b200.h declares, with the reference's parameter defaults.
No compute call is made (there is no GPU here)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*(camr_[a-z0-9_]+)\s*\(",
                            text, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = header_functions()
    for must in ("camr_hydro_umdrv", "camr_level_create", "camr_level_advance",
                 "camr_default_params", "camr_level_get_error"):
        assert must in names


def test_library_exports_every_declared_symbol(native_lib):
    from camr_b200 import native
    names = header_functions()
    missing = [n for n in names if not hasattr(native_lib, n)]
    assert not missing, missing
    # the binding covers every declared entry point too
    assert sorted(native.SIGNATURES) == names


def test_default_params_match_reference_table(native_lib):
    import oracle
    from camr_b200 import native
    p = native.default_params()
    q = oracle.default_params()
    for name, _ in oracle.Params._fields_:
        if name.startswith("pad"):
            continue
        assert getattr(p, name) == getattr(q, name), name
    assert p.riemann_solver == 0
    assert native_lib.camr_version().startswith(b"camr_b200")


def test_invalid_arguments_rejected_without_gpu(native_lib):
    """Argument validation happens before any CUDA call."""
    from camr_b200 import native
    p = native.default_params(cfl=1.5)
    out = C.c_void_p()
    desc = native.LevelDesc()
    st = native_lib.camr_level_create(C.byref(desc), C.byref(p), None, C.byref(out))
    assert native.STATUS[st] == "CAMR_ERR_INVALID"
    p = native.default_params(do_mol=1, cfl=0.5)
    st = native_lib.camr_level_create(C.byref(desc), C.byref(p), None, C.byref(out))
    assert native.STATUS[st] == "CAMR_ERR_INVALID"
    p = native.default_params(riemann_solver=7)
    st = native_lib.camr_level_create(C.byref(desc), C.byref(p), None, C.byref(out))
    assert native.STATUS[st] == "CAMR_ERR_UNSUPPORTED"


def test_batch_tuning_arguments_rejected_without_gpu(native_lib):
    """The launch-shape setters check their arguments before touching a plan."""
    from camr_b200 import native
    ch = (C.c_int * 9)(*([1] * 9))
    gr = (C.c_uint * 9)(*([0] * 9))
    st = native_lib.camr_batch_set_tuning(None, ch, gr, 9)
    assert native.STATUS[st] == "CAMR_ERR_INVALID"
    st = native_lib.camr_batch_tuning(None, ch, gr, 9)
    assert native.STATUS[st] == "CAMR_ERR_INVALID"
    st = native_lib.camr_eb_level_autotune(None)
    assert native.STATUS[st] == "CAMR_ERR_INVALID"


def test_per_box_entry_points_reject_the_same_parameters(native_lib):
    """camr_hydro_umdrv and camr_hydro_umdrv_noalloc validate parameters the
    same way, before any CUDA call (the fab pointers are never read)."""
    from camr_b200 import native
    lo = (C.c_int * 3)(0, 0, 0)
    hi = (C.c_int * 3)(7, 7, 7)
    geom = native.Geom()
    fabs = []
    for _ in range(5):
        f = native.Fab()
        f.ptr = 0x1000  # never dereferenced: the checks fail first
        f.lo = (C.c_int * 3)(-4, -4, -4)
        f.hi = (C.c_int * 3)(11, 11, 11)
        f.ncomp = 10
        fabs.append(f)
    uin, dsdt, fx, fy, fz = fabs
    bad = [dict(cfl=1.5), dict(cfl=0.0), dict(do_mol=1, cfl=0.5), dict(riemann_solver=7),
           dict(do_mol=0, ppm_type=3)]
    for cfg in bad:
        p = native.default_params(**cfg)
        got = []
        for fn in (native_lib.camr_hydro_umdrv, native_lib.camr_hydro_umdrv_noalloc):
            got.append(fn(C.byref(lo), C.byref(hi), C.byref(geom), C.byref(uin), None,
                          C.byref(dsdt), C.byref(fx), C.byref(fy), C.byref(fz), C.byref(p),
                          1e-3, None))
        assert got[0] == got[1] != 0, (cfg, got)
        assert native_lib.camr_noalloc_last_error() != b""
