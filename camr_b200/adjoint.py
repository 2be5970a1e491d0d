"""The hand-written discrete adjoint of the MOL level step behind
torch.autograd (camr_adjoint_* of include/camr_b200.h).

    lev = AdjointLevel(geom, params, checkpoint_every=20)
    S = mol_steps(S0, lev, nsteps)      # S0: CUDA float64 (NVAR, nz, ny, nx)
    J = (S[URHO] * mask).sum() * dV
    J.backward()                         # S0.grad from the library's adjoint

The forward runs on the device through the library (the same kernels as
the level driver); the backward replays each checkpoint segment and reverses
its steps.  The dt sequence is that of the forward run (frozen).  Only
periodic levels with do_mol = 1 are supported; there is no CPU path.
"""
import ctypes as C

import numpy as np

from . import native
from .native import NVAR, check, lib


def _torch():
    import torch
    return torch


class AdjointLevel:
    def __init__(self, geom, params, checkpoint_every=20, stream=None):
        torch = _torch()
        if stream is None:
            stream = torch.cuda.current_stream()
        sp = getattr(stream, "cuda_stream", stream)
        self.geom = geom
        self.n = tuple(geom.dom_hi[d] - geom.dom_lo[d] + 1 for d in range(3))
        h = C.c_void_p()
        check(lib().camr_adjoint_create(C.byref(geom), C.byref(params), int(checkpoint_every),
                                        C.c_void_p(sp), C.byref(h)), "camr_adjoint_create")
        self._h = h
        self.nsteps = 0
        st = C.c_void_p()
        check(lib().camr_adjoint_stream(self._h, C.byref(st)), "camr_adjoint_stream")
        self._stream = torch.cuda.ExternalStream(st.value) if st.value else None

    def _enter(self):
        """Inputs written by torch's current stream must be complete."""
        _torch().cuda.current_stream().synchronize()

    def _leave(self):
        """Outputs must be complete before torch's stream reads them."""
        if self._stream is not None:
            self._stream.synchronize()
        else:
            _torch().cuda.synchronize()

    def close(self):
        if self._h:
            lib().camr_adjoint_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check_state(self, t):
        torch = _torch()
        assert t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()
        assert tuple(t.shape) == (NVAR, self.n[2], self.n[1], self.n[0])

    def forward(self, S0, nsteps, fixed_dts=None):
        torch = _torch()
        self._check_state(S0)
        out = torch.empty_like(S0)
        ptr = None
        if fixed_dts is not None:
            self._dts = np.ascontiguousarray(fixed_dts, dtype=np.float64)
            assert len(self._dts) == nsteps
            ptr = self._dts.ctypes.data
        self._enter()
        check(lib().camr_adjoint_forward(self._h, C.c_void_p(S0.data_ptr()),
                                         C.c_void_p(out.data_ptr()), int(nsteps), ptr),
              "camr_adjoint_forward")
        self._leave()
        self.nsteps = nsteps
        return out

    def backward(self, lam_final):
        torch = _torch()
        lam_final = lam_final.contiguous()
        self._check_state(lam_final)
        out = torch.empty_like(lam_final)
        self._enter()
        check(lib().camr_adjoint_backward(self._h, C.c_void_p(lam_final.data_ptr()),
                                          C.c_void_p(out.data_ptr())), "camr_adjoint_backward")
        self._leave()
        return out

    def dts(self):
        a = (C.c_double * max(self.nsteps, 1))()
        check(lib().camr_adjoint_dts(self._h, a, self.nsteps), "camr_adjoint_dts")
        return np.array(a[:self.nsteps])

    def error(self):
        info = native.ErrorInfo()
        lib().camr_adjoint_get_error(self._h, C.byref(info))
        return (info.code, info.i, info.j, info.k)


def _function():
    torch = _torch()

    class MolSteps(torch.autograd.Function):
        @staticmethod
        def forward(ctx, S0, level, nsteps, fixed_dts):
            ctx.level = level
            return level.forward(S0.detach().contiguous(), nsteps, fixed_dts)

        @staticmethod
        def backward(ctx, grad):
            return ctx.level.backward(grad), None, None, None

    return MolSteps


_FN = None


def mol_steps(S0, level, nsteps, fixed_dts=None):
    """nsteps MOL steps of S0 on `level` (an AdjointLevel), differentiable
    with respect to S0 through the library's adjoint."""
    global _FN
    if _FN is None:
        _FN = _function()
    return _FN.apply(S0, level, nsteps, fixed_dts)
