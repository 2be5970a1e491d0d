"""Host-side mirror of CAMR's hydro call surface over the C ABI.

* :func:`hydro_umdrv` mirrors the per-box ``hydro_umdrv``
  (Source/Hydro/Hydro.H:11-35): Sborder fab in, area-weighted face fluxes and
  an accumulated dSdt out.
* :class:`Level` mirrors one AMR level's ``CAMR::advance`` loop
  (Source/CAMR_advance.cpp:38-164) with Amr's dt logic.

Device memory comes from torch tensors (plumbing only); all arithmetic runs
in libcamr_b200.so.
"""
import ctypes as C

import numpy as np

from . import native
from .native import BC, NVAR, Fab, Geom, LevelDesc, check, default_params, lib

NGROW = 4


def _torch():
    import torch
    return torch


def fab_of(t, lo):
    """Array4 view of a contiguous (ncomp, nz, ny, nx) float64 CUDA tensor."""
    torch = _torch()
    if t.dtype != torch.float64 or not t.is_contiguous() or not t.is_cuda:
        raise ValueError("fab tensors must be contiguous float64 CUDA tensors")
    nc, nz, ny, nx = t.shape
    f = Fab()
    f.ptr = t.data_ptr()
    for d, n in enumerate((nx, ny, nz)):
        f.lo[d] = lo[d]
        f.hi[d] = lo[d] + n - 1
    f.jstride = nx
    f.kstride = nx * ny
    f.nstride = nx * ny * nz
    f.ncomp = nc
    return f


def make_geom(n, dom_lo=(0, 0, 0), is_periodic=(1, 1, 1), bc_lo=(0, 0, 0), bc_hi=(0, 0, 0),
              dx=None, prob_lo=(0.0, 0.0, 0.0), prob_hi=(1.0, 1.0, 1.0)):
    g = Geom()
    for d in range(3):
        g.dom_lo[d] = dom_lo[d]
        g.dom_hi[d] = dom_lo[d] + n[d] - 1
        g.is_periodic[d] = int(is_periodic[d])
        g.bc_lo[d] = BC[bc_lo[d]] if isinstance(bc_lo[d], str) else int(bc_lo[d])
        g.bc_hi[d] = BC[bc_hi[d]] if isinstance(bc_hi[d], str) else int(bc_hi[d])
        g.dx[d] = dx[d] if dx is not None else (prob_hi[d] - prob_lo[d]) / n[d]
        g.prob_lo[d] = prob_lo[d]
    return g


def _stream_ptr(stream):
    if stream is None:
        torch = _torch()
        return torch.cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


def hydro_umdrv(bx_lo, bx_hi, geom, uin, uin_lo, dsdt, flx, params, dt, src=None, stream=None):
    """Per-box hydro (the drop-in for the reference's hydro_umdrv).

    uin: (NVAR, nz, ny, nx) CUDA float64 tensor covering grow(bx,4) starting
    at uin_lo; dsdt: (NVAR, ...) on bx, accumulated; flx: three tensors on
    the faces of bx (overwritten).  Raises CamrError on a non-OK status.
    """
    lo = (C.c_int * 3)(*bx_lo)
    hi = (C.c_int * 3)(*bx_hi)
    fu = fab_of(uin, uin_lo)
    fd = fab_of(dsdt, bx_lo)
    ff = [fab_of(f, bx_lo) for f in flx]
    fs = fab_of(src, uin_lo) if src is not None else None
    st = lib().camr_hydro_umdrv(C.byref(lo), C.byref(hi), C.byref(geom), C.byref(fu),
                                C.byref(fs) if fs is not None else None, C.byref(fd),
                                C.byref(ff[0]), C.byref(ff[1]), C.byref(ff[2]),
                                C.byref(params), float(dt), C.c_void_p(_stream_ptr(stream)))
    check(st, "camr_hydro_umdrv")


def hydro_umdrv_full(bx_lo, bx_hi, geom, uin, uin_lo, q, qaux, dsdt, flx, params, dt,
                     src_q=None, area=None, vol=None, stream=None):
    """The per-box hydro with the reference's full argument list
    (camr_hydro_umdrv_full): q (QVAR) and qaux (5) tensors on grow(bx,4)
    starting at uin_lo, optional src_q (QVAR) likewise, optional face areas
    area[d] (1 comp on the d-faces of bx) and volumes vol (1 comp on bx)."""
    lo = (C.c_int * 3)(*bx_lo)
    hi = (C.c_int * 3)(*bx_hi)
    fu, fq, fa = fab_of(uin, uin_lo), fab_of(q, uin_lo), fab_of(qaux, uin_lo)
    fs = fab_of(src_q, uin_lo) if src_q is not None else None
    fd = fab_of(dsdt, bx_lo)
    ff = [fab_of(f, bx_lo) for f in flx]
    fm = [fab_of(a, bx_lo) for a in area] if area is not None else [None] * 3
    fv = fab_of(vol, bx_lo) if vol is not None else None

    def ref(f):
        return C.byref(f) if f is not None else None

    st = lib().camr_hydro_umdrv_full(C.byref(lo), C.byref(hi), C.byref(geom), C.byref(fu),
                                     C.byref(fq), C.byref(fa), ref(fs), C.byref(fd),
                                     C.byref(ff[0]), C.byref(ff[1]), C.byref(ff[2]), ref(fm[0]),
                                     ref(fm[1]), ref(fm[2]), ref(fv), C.byref(params), float(dt),
                                     C.c_void_p(_stream_ptr(stream)))
    check(st, "camr_hydro_umdrv_full")


def box_fabs(boxes, tensors, ng):
    """camr_box_fab array for boxes [(lo, hi)] and their (NVAR, nz, ny, nx)
    CUDA tensors, each covering its box grown by ng."""
    arr = (native.BoxFab * len(boxes))()
    for b, ((lo, hi), t) in enumerate(zip(boxes, tensors)):
        for d in range(3):
            arr[b].lo[d] = lo[d]
            arr[b].hi[d] = hi[d]
        arr[b].fab = fab_of(t, [lo[d] - ng for d in range(3)])
    return arr


def fill_ghosts(geom, boxes, tensors, ng, stream=None):
    """FillPatch on one level (camr_fill_ghosts): ng ghost layers of every
    box's tensor from the boxes' valid cells and the physical BCs."""
    arr = box_fabs(boxes, tensors, ng)
    check(lib().camr_fill_ghosts(C.byref(geom), len(boxes), arr, int(ng),
                                 C.c_void_p(_stream_ptr(stream))), "camr_fill_ghosts")


def clean_state(geom, boxes, tensors, ng, params, stream=None):
    """clean_state of the boxes with ng ghost layers (camr_clean_state)."""
    arr = box_fabs(boxes, tensors, ng)
    check(lib().camr_clean_state(C.byref(geom), len(boxes), arr, int(ng), C.byref(params),
                                 C.c_void_p(_stream_ptr(stream))), "camr_clean_state")


def est_dt(geom, boxes, tensors, ng, params, stream=None):
    """estTimeStep's hydro dt over the boxes' valid cells (camr_est_dt)."""
    arr = box_fabs(boxes, tensors, ng)
    v = C.c_double()
    check(lib().camr_est_dt(C.byref(geom), len(boxes), arr, C.byref(params), C.byref(v),
                            C.c_void_p(_stream_ptr(stream))), "camr_est_dt")
    return v.value


def get_error(stream=None):
    """Read and clear the library's device error word: (code, i, j, k)."""
    info = native.ErrorInfo()
    lib().camr_get_error(C.c_void_p(_stream_ptr(stream)), C.byref(info))
    return (info.code, info.i, info.j, info.k)


def eb_geometry_to_device(geo, device="cuda"):
    """eb_geometry.sphere_geometry output -> dict of CUDA tensors (kept
    alive by the caller) and the camr_eb_geom struct pointing at them."""
    torch = _torch()
    t = {"flag": torch.from_numpy(geo["flag"].astype(np.int32)).to(device),
         "vfrac": torch.from_numpy(geo["vfrac"]).to(device),
         "ap": [torch.from_numpy(a).to(device) for a in geo["ap"]],
         "fc": [torch.from_numpy(a).contiguous().to(device) for a in geo["fc"]],
         "cent": torch.from_numpy(np.ascontiguousarray(geo["cent"])).to(device)}
    g = native.EBGeom()
    g.flag = t["flag"].data_ptr()
    g.vfrac = t["vfrac"].data_ptr()
    g.cent = t["cent"].data_ptr()
    for d in range(3):
        g.ap[d] = t["ap"][d].data_ptr()
        g.fc[d] = t["fc"][d].data_ptr()
        g.g_lo[d] = geo["lo"][d]
        g.g_hi[d] = geo["hi"][d]
    t["struct"] = g
    return t


def hydro_umdrv_eb(bx_lo, bx_hi, geom, uin, uin_lo, ebdev, params, redist=1, dt=0.0,
                   stream=None):
    """EB per-box hydro on CUDA tensors (MOL, or Godunov-PLM with do_mol = 0):
    uin (NVAR, ...) over a region starting at uin_lo covering grow(bx, 5)
    (MOL) or grow(bx, 6) (Godunov); ebdev from eb_geometry_to_device.
    Returns (dsdt, [flx_x, flx_y, flx_z]) as new CUDA tensors."""
    torch = _torch()
    nb = [bx_hi[d] - bx_lo[d] + 1 for d in range(3)]
    dsdt = torch.zeros((NVAR, nb[2], nb[1], nb[0]), dtype=torch.float64, device=uin.device)
    flx = []
    for d in range(3):
        sh = list(nb)
        sh[d] += 1
        flx.append(torch.zeros((NVAR, sh[2], sh[1], sh[0]), dtype=torch.float64,
                               device=uin.device))
    lo3, hi3 = (C.c_int * 3)(*bx_lo), (C.c_int * 3)(*bx_hi)
    fu = fab_of(uin, uin_lo)
    fd = fab_of(dsdt, bx_lo)
    ff = [fab_of(f, bx_lo) for f in flx]
    check(lib().camr_hydro_umdrv_eb(C.byref(lo3), C.byref(hi3), C.byref(geom), C.byref(fu),
                                    C.byref(ebdev["struct"]), C.byref(fd), C.byref(ff[0]),
                                    C.byref(ff[1]), C.byref(ff[2]), C.byref(params),
                                    int(redist), float(dt), C.c_void_p(_stream_ptr(stream))),
          "camr_hydro_umdrv_eb")
    return dsdt, flx


class Level:
    """One uniform level advanced on the GPU through the C ABI."""

    def __init__(self, geom, params, max_grid_size=(0, 0, 0), use_graph=True, stream=None):
        """stream=None: the library gives the level a non-blocking stream of its own."""
        desc = LevelDesc()
        desc.geom = geom
        for d in range(3):
            desc.max_grid_size[d] = max_grid_size[d]
        desc.use_graph = int(use_graph)
        self.params = params
        self.geom = geom
        self.n = tuple(geom.dom_hi[d] - geom.dom_lo[d] + 1 for d in range(3))
        self.ncell = self.n[0] * self.n[1] * self.n[2]
        sp = None if stream is None else getattr(stream, "cuda_stream", stream)
        h = C.c_void_p()
        check(lib().camr_level_create(C.byref(desc), C.byref(params), C.c_void_p(sp),
                                      C.byref(h)), "camr_level_create")
        self._h = h
        s = C.c_void_p()
        check(lib().camr_level_stream(self._h, C.byref(s)), "camr_level_stream")
        self.stream_ptr = s.value or 0

    def torch_stream(self):
        """The level's stream as a torch stream (for CUDA events)."""
        torch = _torch()
        return torch.cuda.ExternalStream(self.stream_ptr)

    def close(self):
        if self._h:
            lib().camr_level_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, state):
        """state: numpy (host) or CUDA tensor of shape (NVAR, nz, ny, nx)."""
        if isinstance(state, np.ndarray):
            a = np.ascontiguousarray(state, dtype=np.float64)
            assert a.shape == (NVAR, self.n[2], self.n[1], self.n[0])
            check(lib().camr_level_set_state(self._h, a.ctypes.data, 1), "set_state")
            self.sync()
        else:
            assert state.is_cuda and state.is_contiguous()
            check(lib().camr_level_set_state(self._h, state.data_ptr(), 0), "set_state")

    def get_state(self, out=None):
        if out is None:
            out = np.empty((NVAR, self.n[2], self.n[1], self.n[0]))
        if isinstance(out, np.ndarray):
            check(lib().camr_level_get_state(self._h, out.ctypes.data, 1), "get_state")
        else:
            check(lib().camr_level_get_state(self._h, out.data_ptr(), 0), "get_state")
        return out

    def init_finalize(self):
        check(lib().camr_level_init_finalize(self._h), "init_finalize")

    def advance(self, nsteps, fixed_dts=None):
        ptr = None
        if fixed_dts is not None:
            arr = np.ascontiguousarray(fixed_dts, dtype=np.float64)
            assert len(arr) == nsteps
            ptr = arr.ctypes.data
            self._keep = arr
        check(lib().camr_level_advance(self._h, int(nsteps), ptr), "advance")

    def last_dt(self):
        v = C.c_double()
        check(lib().camr_level_last_dt(self._h, C.byref(v)), "last_dt")
        return v.value

    def est_dt(self):
        v = C.c_double()
        check(lib().camr_level_est_dt(self._h, C.byref(v)), "est_dt")
        return v.value

    def error(self):
        info = native.ErrorInfo()
        lib().camr_level_get_error(self._h, C.byref(info))
        return (info.code, info.i, info.j, info.k)

    def restart(self, dt_prev, steps_done):
        """Continue from a checkpoint's state (set_state first): the next dt
        follows computeNewDt against dt_prev."""
        check(lib().camr_level_restart(self._h, float(dt_prev), int(steps_done)), "restart")

    def floor_resets(self):
        """Cells enforce_min_density has reset since the level was created."""
        v = C.c_int64()
        check(lib().camr_level_floor_resets(self._h, C.byref(v)), "floor_resets")
        return v.value

    def sync(self):
        _torch().cuda.synchronize()


class EBLevel:
    """One uniform level with an embedded boundary (MOL, or Godunov-PLM with
    do_mol = 0), advanced on the GPU through camr_eb_level_*.  geo:
    eb_geometry.sphere_geometry output over grow(domain, 5) for MOL,
    grow(domain, 6) for Godunov, one more layer with state redistribution
    (copied into the level).  redist: 1 FluxRedist, 0 NoRedist, 2 StateRedist.
    max_grid_size chops the domain into boxes."""

    def __init__(self, geom, params, geo, redist=1, max_grid_size=(0, 0, 0), use_graph=True,
                 stream=None):
        desc = LevelDesc()
        desc.geom = geom
        for d in range(3):
            desc.max_grid_size[d] = max_grid_size[d]
        desc.use_graph = int(use_graph)
        self.params = params
        self.geom = geom
        self.n = tuple(geom.dom_hi[d] - geom.dom_lo[d] + 1 for d in range(3))
        self.ncell = self.n[0] * self.n[1] * self.n[2]
        host = {"flag": np.ascontiguousarray(geo["flag"], dtype=np.uint32),
                "vfrac": np.ascontiguousarray(geo["vfrac"], dtype=np.float64),
                "ap": [np.ascontiguousarray(a, dtype=np.float64) for a in geo["ap"]],
                "fc": [np.ascontiguousarray(a, dtype=np.float64) for a in geo["fc"]],
                "cent": np.ascontiguousarray(geo["cent"], dtype=np.float64)}
        g = native.EBGeom()
        g.flag = host["flag"].ctypes.data
        g.vfrac = host["vfrac"].ctypes.data
        g.cent = host["cent"].ctypes.data
        for d in range(3):
            g.ap[d] = host["ap"][d].ctypes.data
            g.fc[d] = host["fc"][d].ctypes.data
            g.g_lo[d] = geo["lo"][d]
            g.g_hi[d] = geo["hi"][d]
        sp = None if stream is None else getattr(stream, "cuda_stream", stream)
        h = C.c_void_p()
        check(lib().camr_eb_level_create(C.byref(desc), C.byref(g), C.byref(params),
                                         int(redist), C.c_void_p(sp), C.byref(h)),
              "camr_eb_level_create")
        self._h = h
        s = C.c_void_p()
        check(lib().camr_eb_level_stream(self._h, C.byref(s)), "camr_eb_level_stream")
        self.stream_ptr = s.value or 0

    def torch_stream(self):
        return _torch().cuda.ExternalStream(self.stream_ptr)

    def close(self):
        if self._h:
            lib().camr_eb_level_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, state):
        """state: numpy (host) or CUDA tensor of shape (NVAR, nz, ny, nx)."""
        if isinstance(state, np.ndarray):
            a = np.ascontiguousarray(state, dtype=np.float64)
            assert a.shape == (NVAR, self.n[2], self.n[1], self.n[0])
            check(lib().camr_eb_level_set_state(self._h, a.ctypes.data, 1), "set_state")
            self.sync()
        else:
            assert state.is_cuda and state.is_contiguous()
            check(lib().camr_eb_level_set_state(self._h, state.data_ptr(), 0), "set_state")

    def get_state(self, out=None):
        if out is None:
            out = np.empty((NVAR, self.n[2], self.n[1], self.n[0]))
        if isinstance(out, np.ndarray):
            check(lib().camr_eb_level_get_state(self._h, out.ctypes.data, 1), "get_state")
        else:
            check(lib().camr_eb_level_get_state(self._h, out.data_ptr(), 0), "get_state")
        return out

    def init_finalize(self):
        check(lib().camr_eb_level_init_finalize(self._h), "init_finalize")

    def advance(self, nsteps, fixed_dts=None):
        ptr = None
        if fixed_dts is not None:
            arr = np.ascontiguousarray(fixed_dts, dtype=np.float64)
            assert len(arr) == nsteps
            ptr = arr.ctypes.data
            self._keep = arr
        check(lib().camr_eb_level_advance(self._h, int(nsteps), ptr), "advance")

    def dts(self, n=1 << 16):
        buf = (C.c_double * n)()
        taken = C.c_int()
        check(lib().camr_eb_level_dts(self._h, buf, n, C.byref(taken)), "dts")
        return np.array(buf[:min(taken.value, n)])

    def kernels_per_step(self):
        return int(lib().camr_eb_level_kernels_per_step(self._h))

    def autotune(self):
        check(lib().camr_eb_level_autotune(self._h), "camr_eb_level_autotune")

    def boxes(self):
        r, c, v = C.c_int(), C.c_int(), C.c_int()
        check(lib().camr_eb_level_boxes(self._h, C.byref(r), C.byref(c), C.byref(v)),
              "camr_eb_level_boxes")
        return {"regular": r.value, "cut": c.value, "covered": v.value}

    def floor_resets(self):
        """Cells enforce_min_density has reset since the level was created."""
        v = C.c_int64()
        check(lib().camr_eb_level_floor_resets(self._h, C.byref(v)), "floor_resets")
        return v.value

    def error(self):
        info = native.ErrorInfo()
        lib().camr_eb_level_get_error(self._h, C.byref(info))
        return (info.code, info.i, info.j, info.k)

    def sync(self):
        _torch().cuda.synchronize()


class Batch:
    """A batched hydro plan over the boxes of one level (camr_batch_*).

    boxes: list of (lo, hi, uin, uin_lo, dsdt, flx) with CUDA float64
    tensors as for hydro_umdrv; the tensors must stay alive with the plan.
    """

    PERSISTENT = 0
    PER_BOX = 1

    def __init__(self, boxes, geom, params, stream=None):
        self._keep = boxes
        n = len(boxes)
        tasks = (native.BoxTask * n)()
        for t, (lo, hi, uin, uin_lo, dsdt, flx) in zip(tasks, boxes):
            for d in range(3):
                t.lo[d] = lo[d]
                t.hi[d] = hi[d]
            t.uin = fab_of(uin, uin_lo)
            t.dsdt = fab_of(dsdt, lo)
            for d in range(3):
                t.flx[d] = fab_of(flx[d], lo)
        self._stream = _stream_ptr(stream)
        h = C.c_void_p()
        check(lib().camr_batch_create(n, tasks, C.byref(geom), C.byref(params),
                                      C.c_void_p(self._stream), C.byref(h)), "camr_batch_create")
        self._h = h

    def run(self, dt, mode=PERSISTENT):
        check(lib().camr_batch_run(self._h, float(dt), None, int(mode), C.c_void_p(self._stream)),
              "camr_batch_run")

    def autotune(self, dt):
        check(lib().camr_batch_autotune(self._h, float(dt), C.c_void_p(self._stream)),
              "camr_batch_autotune")

    def tuning(self):
        ch = (C.c_int * 9)()
        gr = (C.c_uint * 9)()
        check(lib().camr_batch_tuning(self._h, ch, gr, 9), "camr_batch_tuning")
        names = ["ctoprim", "flatten_divu", "trace", "flux1", "flux2", "flux3", "mol_slope",
                 "mol_flux", "consup"]
        return {n: (int(c) * 128, int(g)) for n, c, g in zip(names, ch, gr)}

    def set_tuning(self, tuning):
        """Set the launch shapes, as tuning() returns them."""
        names = ["ctoprim", "flatten_divu", "trace", "flux1", "flux2", "flux3", "mol_slope",
                 "mol_flux", "consup"]
        ch = (C.c_int * 9)(*[tuning[n][0] // 128 for n in names])
        gr = (C.c_uint * 9)(*[tuning[n][1] for n in names])
        check(lib().camr_batch_set_tuning(self._h, ch, gr, 9), "camr_batch_set_tuning")

    def close(self):
        if self._h:
            lib().camr_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class AmrHierarchy:
    """Two-level AMR hierarchy (ratio 2, subcycled) advanced on the GPU
    (camr_amr_*): the base level `geom` (periodic) and fine boxes given as
    (lo, hi) fine index triples, coarse-aligned."""

    def __init__(self, geom, params, boxes, max_grid_size=(0, 0, 0), use_graph=True,
                 stream=None):
        desc = LevelDesc()
        desc.geom = geom
        for d in range(3):
            desc.max_grid_size[d] = max_grid_size[d]
        desc.use_graph = int(use_graph)
        self.params = params
        self.geom = geom
        self.boxes = [(tuple(lo), tuple(hi)) for lo, hi in boxes]
        self.n0 = tuple(geom.dom_hi[d] - geom.dom_lo[d] + 1 for d in range(3))
        arr = np.array([list(lo) + list(hi) for lo, hi in self.boxes], dtype=np.int32)
        self._boxes = np.ascontiguousarray(arr)
        sp = None if stream is None else getattr(stream, "cuda_stream", stream)
        h = C.c_void_p()
        check(lib().camr_amr_create(C.byref(desc), len(self.boxes), self._boxes.ctypes.data,
                                    C.byref(params), C.c_void_p(sp), C.byref(h)),
              "camr_amr_create")
        self._h = h
        s = C.c_void_p()
        check(lib().camr_amr_stream(self._h, C.byref(s)), "camr_amr_stream")
        self.stream_ptr = s.value or 0
        self.fine_cells = int(lib().camr_amr_fine_cells(self._h))

    def torch_stream(self):
        return _torch().cuda.ExternalStream(self.stream_ptr)

    def close(self):
        if self._h:
            lib().camr_amr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, S0, S1):
        """S0: (NVAR, nz, ny, nx) base state; S1: the fine boxes' states back
        to back (flat), numpy (host) or CUDA tensors."""
        if isinstance(S0, np.ndarray):
            a = np.ascontiguousarray(S0, dtype=np.float64)
            b = np.ascontiguousarray(S1, dtype=np.float64)
            assert a.size == NVAR * self.n0[0] * self.n0[1] * self.n0[2]
            assert b.size == NVAR * self.fine_cells
            check(lib().camr_amr_set_state(self._h, a.ctypes.data, b.ctypes.data, 1),
                  "camr_amr_set_state")
            self.sync()
        else:
            check(lib().camr_amr_set_state(self._h, S0.data_ptr(), S1.data_ptr(), 0),
                  "camr_amr_set_state")

    def get_state(self, S0=None, S1=None):
        if S0 is None:
            S0 = np.empty((NVAR, self.n0[2], self.n0[1], self.n0[0]))
            S1 = np.empty(NVAR * self.fine_cells)
        if isinstance(S0, np.ndarray):
            check(lib().camr_amr_get_state(self._h, S0.ctypes.data, S1.ctypes.data, 1),
                  "camr_amr_get_state")
        else:
            check(lib().camr_amr_get_state(self._h, S0.data_ptr(), S1.data_ptr(), 0),
                  "camr_amr_get_state")
        return S0, S1

    def init_finalize(self):
        check(lib().camr_amr_init_finalize(self._h), "camr_amr_init_finalize")

    def advance(self, nsteps):
        check(lib().camr_amr_advance(self._h, int(nsteps)), "camr_amr_advance")

    def clock(self):
        c = (C.c_double * 4)()
        check(lib().camr_amr_clock(self._h, c), "camr_amr_clock")
        return list(c)

    def restart(self, clock, steps_done):
        """Continue from a checkpoint's states (set_state first): clock =
        (t0, t1, dt0, dt1) as clock() returns it."""
        c = (C.c_double * 4)(*clock)
        check(lib().camr_amr_restart(self._h, C.byref(c), int(steps_done)), "amr restart")

    def floor_resets(self):
        """Cells enforce_min_density has reset on either level so far."""
        v = C.c_int64()
        check(lib().camr_amr_floor_resets(self._h, C.byref(v)), "floor_resets")
        return v.value

    def autotune(self):
        check(lib().camr_amr_autotune(self._h), "camr_amr_autotune")

    PERSISTENT = 0
    PER_BOX = 1

    def set_fine_mode(self, mode):
        check(lib().camr_amr_set_fine_mode(self._h, int(mode)), "camr_amr_set_fine_mode")

    def kernels_per_step(self):
        return int(lib().camr_amr_kernels_per_step(self._h))

    def error(self):
        info = native.ErrorInfo()
        lib().camr_amr_get_error(self._h, C.byref(info))
        return (info.code, info.i, info.j, info.k)

    def sync(self):
        _torch().cuda.synchronize()


def level_boxes(n, max_grid_size, dom_lo=(0, 0, 0)):
    """The domain chopped by max_grid_size from the low end (0 = one box),
    as a list of (lo, hi) tuples in i-fastest order."""
    step = [max_grid_size[d] if max_grid_size[d] > 0 else n[d] for d in range(3)]
    out = []
    for k in range(dom_lo[2], dom_lo[2] + n[2], step[2]):
        for j in range(dom_lo[1], dom_lo[1] + n[1], step[1]):
            for i in range(dom_lo[0], dom_lo[0] + n[0], step[0]):
                lo = (i, j, k)
                hi = tuple(min(lo[d] + step[d] - 1, dom_lo[d] + n[d] - 1) for d in range(3))
                out.append((lo, hi))
    return out


def write_plotfile(path, state, geom, prob_hi, time=0.0, level_step=0,
                   max_grid_size=(32, 32, 32), comps=None, names=None):
    """Write one level's state (numpy (NVAR, nz, ny, nx), valid cells) as an
    AMReX plotfile directory (camr_write_plotfile)."""
    n = tuple(geom.dom_hi[d] - geom.dom_lo[d] + 1 for d in range(3))
    a = np.ascontiguousarray(state, dtype=np.float64)
    assert a.shape == (NVAR, n[2], n[1], n[0])
    boxes = level_boxes(n, max_grid_size, tuple(geom.dom_lo))
    flat = np.array([list(lo) + list(hi) for lo, hi in boxes], dtype=np.int32).ravel()
    comps = list(range(NVAR)) if comps is None else list(comps)
    carr = np.array(comps, dtype=np.int32)
    nm = None
    if names is not None:
        nm = (C.c_char_p * len(names))(*[x.encode() for x in names])
    ph = (C.c_double * 3)(*prob_hi)
    st = lib().camr_write_plotfile(str(path).encode(), C.byref(geom), C.byref(ph), float(time),
                                   int(level_step), len(boxes), flat.ctypes.data, a.ctypes.data,
                                   len(comps), carr.ctypes.data, nm)
    if st != 0:
        raise native.CamrError(st, "camr_write_plotfile " +
                               lib().camr_io_last_error().decode())


def write_plotfile_amr(path, S0, S1, geom, prob_hi, fine_boxes, time=0.0, level_steps=(0, 0),
                       max_grid_size=(32, 32, 32), comps=None, names=None):
    """Write the two levels of an AMR run as one plotfile
    (camr_write_plotfile_amr): S0 the base level (NVAR, nz, ny, nx); S1 the
    fine boxes' states back to back (each (NVAR, nz, ny, nx) over its box, as
    AmrHierarchy.get_state returns them); fine_boxes [(lo, hi), ...] on the fine
    index space."""
    n = tuple(geom.dom_hi[d] - geom.dom_lo[d] + 1 for d in range(3))
    a = np.ascontiguousarray(S0, dtype=np.float64)
    assert a.shape == (NVAR, n[2], n[1], n[0])
    f = np.ascontiguousarray(S1, dtype=np.float64).ravel()
    ncell1 = sum((h[0] - l[0] + 1) * (h[1] - l[1] + 1) * (h[2] - l[2] + 1) for l, h in fine_boxes)
    assert f.size == NVAR * ncell1
    boxes0 = level_boxes(n, max_grid_size, tuple(geom.dom_lo))
    b0 = np.array([list(lo) + list(hi) for lo, hi in boxes0], dtype=np.int32).ravel()
    b1 = np.array([list(lo) + list(hi) for lo, hi in fine_boxes], dtype=np.int32).ravel()
    comps = list(range(NVAR)) if comps is None else list(comps)
    carr = np.array(comps, dtype=np.int32)
    nm = None
    if names is not None:
        nm = (C.c_char_p * len(names))(*[x.encode() for x in names])
    ph = (C.c_double * 3)(*prob_hi)
    steps = (C.c_int * 2)(*level_steps)
    st = lib().camr_write_plotfile_amr(str(path).encode(), C.byref(geom), C.byref(ph), float(time),
                                       steps, len(boxes0), b0.ctypes.data, a.ctypes.data,
                                       len(fine_boxes), b1.ctypes.data if len(fine_boxes) else None,
                                       f.ctypes.data, len(comps), carr.ctypes.data, nm)
    if st != 0:
        raise native.CamrError(st, "camr_write_plotfile_amr " +
                               lib().camr_io_last_error().decode())


def write_checkpoint(path, geom, prob_hi, S0, time, dt, level_step, S1=None, fine_boxes=(),
                     max_grid_size=(32, 32, 32), cpu_time=0.0):
    """Checkpoint of one level (S0) or of the two-level hierarchy (S0, S1,
    fine_boxes) in CAMR::checkPoint's layout (camr_write_checkpoint).  time,
    dt, level_step: per level (a number for one level)."""
    n = tuple(geom.dom_hi[d] - geom.dom_lo[d] + 1 for d in range(3))
    a = np.ascontiguousarray(S0, dtype=np.float64)
    assert a.shape == (NVAR, n[2], n[1], n[0])
    boxes0 = level_boxes(n, max_grid_size, tuple(geom.dom_lo))
    b0 = np.array([list(lo) + list(hi) for lo, hi in boxes0], dtype=np.int32).ravel()
    two = len(fine_boxes) > 0
    f = np.ascontiguousarray(S1, dtype=np.float64).ravel() if two else None
    b1 = (np.array([list(lo) + list(hi) for lo, hi in fine_boxes], dtype=np.int32).ravel()
          if two else None)
    per = (lambda v: tuple(v) if np.ndim(v) else (v, 0))  # noqa: E731
    t = (C.c_double * 2)(*per(time))
    d = (C.c_double * 2)(*per(dt))
    stp = (C.c_int * 2)(*[int(x) for x in per(level_step)])
    ph = (C.c_double * 3)(*prob_hi)
    st = lib().camr_write_checkpoint(str(path).encode(), C.byref(geom), C.byref(ph), C.byref(t),
                                     C.byref(d), C.byref(stp), len(boxes0), b0.ctypes.data,
                                     a.ctypes.data, len(fine_boxes),
                                     b1.ctypes.data if two else None,
                                     f.ctypes.data if two else None, float(cpu_time))
    if st != 0:
        raise native.CamrError(st, "camr_write_checkpoint " + lib().camr_io_last_error().decode())


def read_checkpoint(path, geom, fine_boxes=()):
    """Read a checkpoint of write_checkpoint back: (S0, S1 or None, times,
    dts, level steps), the per-level values as tuples."""
    n = tuple(geom.dom_hi[d] - geom.dom_lo[d] + 1 for d in range(3))
    s0 = np.zeros((NVAR, n[2], n[1], n[0]))
    ncell1 = sum((h[0] - l[0] + 1) * (h[1] - l[1] + 1) * (h[2] - l[2] + 1) for l, h in fine_boxes)
    two = len(fine_boxes) > 0
    s1 = np.zeros(NVAR * ncell1) if two else None
    b1 = (np.array([list(lo) + list(hi) for lo, hi in fine_boxes], dtype=np.int32).ravel()
          if two else None)
    t = (C.c_double * 2)()
    d = (C.c_double * 2)()
    stp = (C.c_int * 2)()
    st = lib().camr_read_checkpoint(str(path).encode(), C.byref(geom), C.byref(t), C.byref(d),
                                    C.byref(stp), s0.ctypes.data, len(fine_boxes),
                                    b1.ctypes.data if two else None,
                                    s1.ctypes.data if two else None)
    if st != 0:
        raise native.CamrError(st, "camr_read_checkpoint " + lib().camr_io_last_error().decode())
    nl = 2 if two else 1
    return s0, s1, tuple(t)[:nl], tuple(d)[:nl], tuple(stp)[:nl]


def read_plotfile_amr(path, geom, fine_boxes, ncomp=NVAR):
    """Read a plotfile of write_plotfile_amr back for the hierarchy with
    these fine boxes: returns (S0 (ncomp, nz, ny, nx), S1 flat in the
    AmrHierarchy.set_state layout, time, (step0, step1))."""
    n = tuple(geom.dom_hi[d] - geom.dom_lo[d] + 1 for d in range(3))
    s0 = np.zeros((ncomp, n[2], n[1], n[0]))
    ncell1 = sum((h[0] - l[0] + 1) * (h[1] - l[1] + 1) * (h[2] - l[2] + 1) for l, h in fine_boxes)
    s1 = np.zeros(NVAR * ncell1)
    b1 = np.array([list(lo) + list(hi) for lo, hi in fine_boxes], dtype=np.int32).ravel()
    t = C.c_double()
    steps = (C.c_int * 2)()
    st = lib().camr_read_plotfile_amr(str(path).encode(), C.byref(geom), int(ncomp),
                                      s0.ctypes.data, len(fine_boxes),
                                      b1.ctypes.data if len(fine_boxes) else None,
                                      s1.ctypes.data if len(fine_boxes) else None, C.byref(t),
                                      steps)
    if st != 0:
        raise native.CamrError(st, "camr_read_plotfile_amr " +
                               lib().camr_io_last_error().decode())
    return s0, s1, t.value, (steps[0], steps[1])


def read_plotfile(path, geom, ncomp=NVAR):
    """Read a single-level plotfile written by write_plotfile: returns
    (state planes (ncomp, nz, ny, nx), time, level_step)."""
    n = tuple(geom.dom_hi[d] - geom.dom_lo[d] + 1 for d in range(3))
    out = np.zeros((ncomp, n[2], n[1], n[0]))
    t = C.c_double()
    stp = C.c_int()
    st = lib().camr_read_plotfile(str(path).encode(), C.byref(geom), int(ncomp),
                                  out.ctypes.data, C.byref(t), C.byref(stp))
    if st != 0:
        raise native.CamrError(st, "camr_read_plotfile " + lib().camr_io_last_error().decode())
    return out, t.value, stp.value
