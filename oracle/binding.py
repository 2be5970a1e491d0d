"""ctypes binding of the oracle libraries (see oracle_abi.h)."""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NVAR, QVAR, NGDNV = 10, 11, 6
_LIBS = {}


def lib_path_eb():
    return os.path.join(HERE, "_ref", "libcamr_ref_eb.so")


_EB = None


def load_eb():
    """The reference's EB hydro (oracle/_ref/libcamr_ref_eb.so)."""
    global _EB
    if _EB is None:
        path = lib_path_eb()
        if not os.path.exists(path):
            raise FileNotFoundError(f"EB oracle library missing: {path} (run `make -C oracle ref`)")
        lib = C.CDLL(path)
        lib.orc_hydro_box_eb.restype = C.c_long
        _EB = lib
    return _EB


def hydro_box_eb(p, bx_lo, bx_hi, dom_lo, dom_hi, bclo, bchi, periodic, uin, g_lo, geo, dx, dt,
                 redist=1, weights_type=2):
    """Per-box EB hydro (MOL, or Godunov with p.do_mol = 0).  uin: (NVAR, ...)
    over G = [g_lo, g_lo + shape - 1]; geo: eb_geometry.sphere_geometry
    output over the same G.  redist: 0 none, 1 flux, 2 state redistribution.
    Returns
    (dsdt on bx, [flx_x, flx_y, flx_z] on bx faces, nassert)."""
    lib = load_eb()
    nb = [bx_hi[d] - bx_lo[d] + 1 for d in range(3)]
    uin = np.ascontiguousarray(uin, dtype=np.float64)
    g_hi = [g_lo[d] + uin.shape[3 - d] - 1 for d in range(3)]
    dsdt = np.zeros((NVAR, nb[2], nb[1], nb[0]))
    flx = []
    for d in range(3):
        s = list(nb)
        s[d] += 1
        flx.append(np.zeros((NVAR, s[2], s[1], s[0])))
    I3 = _I3
    arr = [np.ascontiguousarray(a, dtype=np.float64) for a in geo["ap"]]
    fcs = [np.ascontiguousarray(a, dtype=np.float64) for a in geo["fc"]]
    flag = np.ascontiguousarray(geo["flag"], dtype=np.uint32)
    vf = np.ascontiguousarray(geo["vfrac"], dtype=np.float64)
    P = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    cent = np.ascontiguousarray(geo["cent"], dtype=np.float64)
    n = lib.orc_hydro_box_eb(C.byref(p), I3(*bx_lo), I3(*bx_hi), I3(*dom_lo), I3(*dom_hi),
                             I3(*bclo), I3(*bchi), I3(*periodic), P(uin), I3(*g_lo), I3(*g_hi),
                             P(flag), P(vf), P(arr[0]), P(arr[1]), P(arr[2]), P(fcs[0]),
                             P(fcs[1]), P(fcs[2]), P(cent), int(redist), int(weights_type),
                             P(dsdt), P(flx[0]), P(flx[1]), P(flx[2]), _D3(*dx),
                             C.c_double(dt))
    return dsdt, flx, n


def eb_advance(p, lev, geo, state, nsteps, first_step=True, dt_prev=0.0, redist=1):
    """EB level steps (MOL) on the whole domain as one box.  geo: geometry
    over grow(domain, 5); state (NVAR, nz, ny, nx) updated in place.
    Returns (dt_last, dt_hist, nassert)."""
    lib = load_eb()
    if not hasattr(lib, "_eb_adv_ready"):
        lib.orc_eb_advance.restype = C.c_long
        lib._eb_adv_ready = True
    assert state.dtype == np.float64 and state.flags["C_CONTIGUOUS"]
    arr = [np.ascontiguousarray(a, dtype=np.float64) for a in geo["ap"]]
    fcs = [np.ascontiguousarray(a, dtype=np.float64) for a in geo["fc"]]
    flag = np.ascontiguousarray(geo["flag"], dtype=np.uint32)
    vf = np.ascontiguousarray(geo["vfrac"], dtype=np.float64)
    P = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    dtp = C.c_double(dt_prev)
    hist = np.zeros(max(nsteps, 1))
    cent = np.ascontiguousarray(geo["cent"], dtype=np.float64)
    n = lib.orc_eb_advance(C.byref(p), C.byref(lev), P(flag), P(vf), P(arr[0]), P(arr[1]),
                           P(arr[2]), P(fcs[0]), P(fcs[1]), P(fcs[2]), P(cent), P(state), int(nsteps),
                           int(bool(first_step)), C.byref(dtp), P(hist), int(redist))
    return dtp.value, hist[:nsteps], n


def eb_init_finalize(p, lev, state):
    """initData's epilogue with the EB guards on state (NVAR, nz, ny, nx)."""
    lib = load_eb()
    assert state.dtype == np.float64 and state.flags["C_CONTIGUOUS"]
    lib.orc_eb_init_finalize(C.byref(p), C.byref(lev), state.ctypes.data_as(C.c_void_p))


def lib_path(kind):
    if kind == "restate":
        return os.path.join(HERE, "_lib", "libcamr_oracle.so")
    if kind == "ref":
        return os.path.join(HERE, "_ref", "libcamr_ref.so")
    raise ValueError(kind)


def build(ref=None, ref_src=None):
    """Build the restatement, and the reference library from the reference
    checkout's Source/ directory: `ref_src`, else $CAMR_REF_SRC.  ref=None
    builds the reference library when such a directory is given and exists;
    ref=True without one is an error."""
    subprocess.run(["make", "-C", HERE, "all"], check=True)
    src = ref_src or os.environ.get("CAMR_REF_SRC")
    if ref is None:
        ref = bool(src) and os.path.isdir(src)
    if ref:
        if not src:
            raise RuntimeError("building the reference library needs its Source/ directory: "
                               "pass ref_src= or set CAMR_REF_SRC")
        subprocess.run(["make", "-C", HERE, "ref", f"REF_SRC={src}"], check=True)


class Params(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "do_mol", "ppm_type", "plm_iorder", "use_pslope", "use_flattening",
        "transverse_reset_density", "dual_energy_update_E_from_e",
        "allow_negative_energy", "allow_small_energy", "add_grav_src",
        "eb_weights_type", "riemann_solver")] + [(n, C.c_double) for n in (
        "difmag", "small", "small_dens", "small_temp", "small_pres",
        "dual_energy_eta1", "dual_energy_eta2", "const_grav", "cfl",
        "init_shrink", "change_max", "fixed_dt", "initial_dt", "max_dt",
        "eos_gamma", "smallu", "small_num")]


class Level(C.Structure):
    _fields_ = [("dom_lo", C.c_int * 3), ("dom_hi", C.c_int * 3),
                ("is_periodic", C.c_int * 3), ("bc_lo", C.c_int * 3),
                ("bc_hi", C.c_int * 3), ("max_grid_size", C.c_int * 3),
                ("tile_size", C.c_int * 3), ("nthreads", C.c_int),
                ("dx", C.c_double * 3)]


_I3 = C.c_int * 3
_D3 = C.c_double * 3
_DP = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def load(kind="restate"):
    if kind in _LIBS:
        return _LIBS[kind]
    path = lib_path(kind)
    if not os.path.exists(path):
        raise FileNotFoundError(f"oracle library missing: {path} (run `make -C oracle`)")
    lib = C.CDLL(path)
    lib.orc_hydro_box.restype = C.c_long
    lib.orc_hydro_box.argtypes = [
        C.POINTER(Params), _I3, _I3, _I3, _I3, _I3, _I3, _DP, _I3, _I3,
        C.c_void_p, _DP, _I3, _I3, _DP, _DP, _DP, _D3, C.c_double]
    lib.orc_default_params.argtypes = [C.POINTER(Params)]
    lib.orc_init_finalize.argtypes = [C.POINTER(Params), C.POINTER(Level), _DP]
    lib.orc_est_dt.restype = C.c_double
    lib.orc_est_dt.argtypes = [C.POINTER(Params), C.POINTER(Level), _DP]
    lib.orc_advance.restype = C.c_long
    lib.orc_advance.argtypes = [C.POINTER(Params), C.POINTER(Level), _DP, C.c_int,
                                C.c_int, C.POINTER(C.c_double), C.c_void_p]
    lib.orc_advance_fixed_dt.restype = C.c_long
    lib.orc_advance_fixed_dt.argtypes = [C.POINTER(Params), C.POINTER(Level), _DP,
                                         C.c_int, _DP]
    lib.orc_expand_state.argtypes = [C.POINTER(Params), C.POINTER(Level), _DP, C.c_int, _DP]
    lib.orc_clean_state.argtypes = [C.POINTER(Params), C.POINTER(Level), _DP]
    lib.orc_amr_run.restype = C.c_long
    lib.orc_amr_run.argtypes = [C.POINTER(Params), C.POINTER(Level), C.c_int, C.c_void_p,
                                _DP, _DP, C.c_int, C.c_int, C.c_int, _DP, C.c_void_p]
    lib.orc_fluxreg_reflux.restype = None
    lib.orc_fluxreg_reflux.argtypes = [C.POINTER(Level), C.c_int, C.c_void_p, C.c_int, _DP,
                                       C.c_double,
                                       C.c_int, C.c_void_p, C.c_int, _DP, C.c_double, _DP]
    lib.orc_fine_fill_ghosts.restype = None
    lib.orc_fine_fill_ghosts.argtypes = [C.POINTER(Level), C.c_int, C.c_void_p, _DP, _DP, _DP,
                                         C.c_double, C.c_double, C.c_double]
    lib.orc_avg_down.restype = None
    lib.orc_avg_down.argtypes = [C.POINTER(Level), C.c_int, C.c_void_p, _DP, _DP]
    _LIBS[kind] = lib
    return lib


def default_params(**kw):
    p = Params()
    load("restate").orc_default_params(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def make_level(n, lo=(0, 0, 0), periodic=(1, 1, 1), bc_lo=(0, 0, 0), bc_hi=(0, 0, 0),
               dx=None, max_grid_size=(0, 0, 0), tile_size=(0, 0, 0), nthreads=None,
               prob_len=(1.0, 1.0, 1.0)):
    lev = Level()
    for d in range(3):
        lev.dom_lo[d] = lo[d]
        lev.dom_hi[d] = lo[d] + n[d] - 1
        lev.is_periodic[d] = periodic[d]
        lev.bc_lo[d] = bc_lo[d]
        lev.bc_hi[d] = bc_hi[d]
        lev.max_grid_size[d] = max_grid_size[d]
        lev.tile_size[d] = tile_size[d]
        lev.dx[d] = dx[d] if dx is not None else prob_len[d] / n[d]
    lev.nthreads = nthreads or os.cpu_count() or 1
    return lev


def hydro_box(kind, p, bx_lo, bx_hi, dom_lo, dom_hi, bclo, bchi, uin, uin_lo, dx, dt,
              src=None, dsdt_init=None):
    """Per-box hydro; returns (dsdt on bx, [flx_x, flx_y, flx_z], nassert)."""
    lib = load(kind)
    bx_lo, bx_hi = list(bx_lo), list(bx_hi)
    nb = [bx_hi[d] - bx_lo[d] + 1 for d in range(3)]
    uin = np.ascontiguousarray(uin, dtype=np.float64)
    uin_hi = [uin_lo[d] + uin.shape[3 - d] - 1 for d in range(3)]
    dsdt = np.zeros((NVAR, nb[2], nb[1], nb[0]))
    if dsdt_init is not None:
        dsdt[...] = dsdt_init
    flx = []
    for d in range(3):
        s = list(nb)
        s[d] += 1
        flx.append(np.zeros((NVAR, s[2], s[1], s[0])))
    srcp = None
    if src is not None:
        src = np.ascontiguousarray(src, dtype=np.float64)
        srcp = src.ctypes.data
    nass = lib.orc_hydro_box(C.byref(p), _I3(*bx_lo), _I3(*bx_hi), _I3(*dom_lo),
                             _I3(*dom_hi), _I3(*bclo), _I3(*bchi), uin, _I3(*uin_lo),
                             _I3(*uin_hi), srcp, dsdt, _I3(*bx_lo), _I3(*bx_hi),
                             flx[0], flx[1], flx[2], _D3(*dx), float(dt))
    return dsdt, flx, nass


def lib_path_flops():
    return os.path.join(HERE, "_ref", "libcamr_ref_flops.so")


def count_flops(p, n, bclo, bchi, uin, dx, dt):
    """Operations of the reference's per-box hydro (ctoprim, srctoprim,
    hydro_umdrv) on the box [0, n-1] with uin (NVAR, n2+8, n1+8, n0+8) on
    grow(box, 4): dict of adds, muls, divs, sqrts, cmps, other (abs /
    copysign) and flops = adds + muls + divs + sqrts."""
    lib = C.CDLL(lib_path_flops())
    lib.orc_count_flops.restype = C.c_long
    uin = np.ascontiguousarray(uin, dtype=np.float64)
    assert uin.shape == (NVAR, n[2] + 8, n[1] + 8, n[0] + 8)
    c = (C.c_longlong * 6)()
    nass = lib.orc_count_flops(C.byref(p), _I3(*n), _I3(*bclo), _I3(*bchi),
                               C.c_void_p(uin.ctypes.data), _D3(*dx), C.c_double(dt), c)
    assert nass == 0
    names = ["adds", "muls", "divs", "sqrts", "cmps", "other"]
    out = {k: int(v) for k, v in zip(names, c)}
    out["flops"] = out["adds"] + out["muls"] + out["divs"] + out["sqrts"]
    return out


def ref_ctoprim(p, lo, hi, uin, uin_lo, src=None):
    """The reference's hydro_ctoprim / hydro_srctoprim over [lo, hi] of uin
    (oracle/_ref only): (q (QVAR, ...), qaux (5, ...), src_q (QVAR, ...))."""
    lib = load("ref")
    lib.orc_ref_ctoprim.restype = C.c_long
    n = [hi[d] - lo[d] + 1 for d in range(3)]
    uin = np.ascontiguousarray(uin, dtype=np.float64)
    uin_hi = [uin_lo[d] + uin.shape[3 - d] - 1 for d in range(3)]
    q = np.zeros((QVAR, n[2], n[1], n[0]))
    qaux = np.zeros((5, n[2], n[1], n[0]))
    srcq = np.zeros((QVAR, n[2], n[1], n[0]))
    srcp = None
    if src is not None:
        src = np.ascontiguousarray(src, dtype=np.float64)
        srcp = src.ctypes.data
    vp = C.c_void_p
    nass = lib.orc_ref_ctoprim(C.byref(p), _I3(*lo), _I3(*hi), vp(uin.ctypes.data), _I3(*uin_lo),
                               _I3(*uin_hi), vp(srcp), vp(q.ctypes.data), vp(qaux.ctypes.data),
                               vp(srcq.ctypes.data))
    assert nass == 0
    return q, qaux, srcq


def ref_hydro_box_full(p, bx_lo, bx_hi, dom_lo, dom_hi, bclo, bchi, uin, uin_lo, q, qaux, srcq,
                       area, vol, dx, dt):
    """The reference's hydro_umdrv with caller q/qaux/src_q and metrics
    (oracle/_ref only); returns (dsdt, [flx_x, flx_y, flx_z], nassert)."""
    lib = load("ref")
    lib.orc_ref_hydro_box_full.restype = C.c_long
    nb = [bx_hi[d] - bx_lo[d] + 1 for d in range(3)]
    uin = np.ascontiguousarray(uin, dtype=np.float64)
    uin_hi = [uin_lo[d] + uin.shape[3 - d] - 1 for d in range(3)]
    dsdt = np.zeros((NVAR, nb[2], nb[1], nb[0]))
    flx = []
    for d in range(3):
        s = list(nb)
        s[d] += 1
        flx.append(np.zeros((NVAR, s[2], s[1], s[0])))
    keep = []

    def ptr(a):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=np.float64)
        keep.append(a)
        return C.c_void_p(a.ctypes.data)

    areas = list(area) if area is not None else [None, None, None]
    nass = lib.orc_ref_hydro_box_full(
        C.byref(p), _I3(*bx_lo), _I3(*bx_hi), _I3(*dom_lo), _I3(*dom_hi), _I3(*bclo), _I3(*bchi),
        ptr(uin), _I3(*uin_lo), _I3(*uin_hi), ptr(q), ptr(qaux), ptr(srcq), ptr(areas[0]),
        ptr(areas[1]), ptr(areas[2]), ptr(vol), ptr(dsdt), ptr(flx[0]), ptr(flx[1]), ptr(flx[2]),
        _D3(*dx), C.c_double(dt))
    return dsdt, flx, nass


def init_finalize(kind, p, lev, state):
    load(kind).orc_init_finalize(C.byref(p), C.byref(lev), state)


def est_dt(kind, p, lev, state):
    return load(kind).orc_est_dt(C.byref(p), C.byref(lev), np.ascontiguousarray(state))


def advance(kind, p, lev, state, nsteps, first_step=True, dt_prev=0.0):
    """Advance in place; returns (dt_last, dt_history, nassert)."""
    hist = np.zeros(nsteps)
    dtp = C.c_double(dt_prev)
    n = load(kind).orc_advance(C.byref(p), C.byref(lev), state, nsteps, int(first_step),
                               C.byref(dtp), hist.ctypes.data)
    return dtp.value, hist, n


def advance_fixed_dt(kind, p, lev, state, dts):
    dts = np.ascontiguousarray(dts, dtype=np.float64)
    return load(kind).orc_advance_fixed_dt(C.byref(p), C.byref(lev), state, len(dts), dts)


def expand_state(kind, p, lev, state, ng=4):
    n = [lev.dom_hi[d] - lev.dom_lo[d] + 1 for d in range(3)]
    border = np.zeros((NVAR, n[2] + 2 * ng, n[1] + 2 * ng, n[0] + 2 * ng))
    load(kind).orc_expand_state(C.byref(p), C.byref(lev), np.ascontiguousarray(state), ng,
                                border)
    return border


def clean_state(kind, p, lev, state):
    load(kind).orc_clean_state(C.byref(p), C.byref(lev), state)


def amr_run(kind, p, lev0, boxes, S0, S1, nsteps, do_init=False, first_step=True,
            clock=None):
    """Two-level run in place.  boxes: (nbox, 6) int array of fine lo/hi;
    S0: coarse valid state; S1: 1-D array, the fine boxes' states back to
    back; clock: float64[4] (times of both levels, last dt of both levels),
    updated in place.  Returns (dt history (nsteps, 2), nassert)."""
    boxes = np.ascontiguousarray(boxes, dtype=np.int32).reshape(-1, 6)
    hist = np.zeros((max(nsteps, 1), 2))
    if clock is None:
        clock = np.zeros(4)
    n = load(kind).orc_amr_run(C.byref(p), C.byref(lev0), len(boxes), boxes.ctypes.data,
                               S0, S1, nsteps, int(do_init), int(first_step), clock,
                               hist.ctypes.data)
    return hist[:nsteps], n


def fluxreg_reflux(kind, lev0, cboxes, cflux, dtdx_c, fboxes, fflux, dtdx_f, S0):
    """The restated two-level flux register on given fluxes, S0 refluxed in
    place (orc_fluxreg_reflux).  cboxes / fboxes: (n, 6) lo/hi of the
    coarse and fine boxes; cflux[call][c][d]: NVAR x faces(coarse box c, d)
    arrays (component slowest, i fastest) of each coarse hydro call;
    fflux[call][b][d]: the same for fine box b in each fine hydro call."""
    cb = np.ascontiguousarray(cboxes, dtype=np.int32).reshape(-1, 6)
    fb = np.ascontiguousarray(fboxes, dtype=np.int32).reshape(-1, 6)
    cf = np.ascontiguousarray(np.concatenate([np.ravel(a) for call in cflux for per in call
                                              for a in per]))
    ff = (np.ascontiguousarray(np.concatenate([np.ravel(a) for call in fflux for per in call
                                                for a in per]))
          if fflux else np.zeros(1))
    load(kind).orc_fluxreg_reflux(C.byref(lev0), len(cb), cb.ctypes.data, len(cflux), cf,
                                  float(dtdx_c),
                                  len(fb), fb.ctypes.data, len(fflux), ff, float(dtdx_f), S0)


def avg_down(kind, lev0, fboxes, fine_states, S0):
    """The restated avgDown (orc_avg_down): S0's covered cells from the fine
    boxes' states (fine_states[b]: NVAR x box, component slowest), in
    place."""
    fb = np.ascontiguousarray(fboxes, dtype=np.int32).reshape(-1, 6)
    s1 = np.ascontiguousarray(np.concatenate([np.ravel(a) for a in fine_states]))
    load(kind).orc_avg_down(C.byref(lev0), len(fb), fb.ctypes.data, s1, S0)


def fine_fill_ghosts(kind, lev0, fboxes, grown, c_old, c_new, t0, t1, t):
    """The restated two-level ghost fill (orc_fine_fill_ghosts) of the fine
    boxes' grown-by-4 states grown[b] (NVAR x grown box, valid cells set),
    from the coarse states c_old / c_new at times t0 / t1, for time t.
    Returns the filled arrays."""
    fb = np.ascontiguousarray(fboxes, dtype=np.int32).reshape(-1, 6)
    sizes = [a.size for a in grown]
    flat = np.ascontiguousarray(np.concatenate([np.ravel(a) for a in grown]))
    load(kind).orc_fine_fill_ghosts(C.byref(lev0), len(fb), fb.ctypes.data, flat,
                                    np.ascontiguousarray(c_old), np.ascontiguousarray(c_new),
                                    float(t0), float(t1), float(t))
    out, at = [], 0
    for a, k in zip(grown, sizes):
        out.append(flat[at:at + k].reshape(a.shape))
        at += k
    return out
