"""GPU tests of the hand-written discrete adjoint (camr_adjoint_*,
camr_b200.adjoint):

* its forward pass gives the level driver's bits and dt sequence;
* its gradient equals the taped FP64 CPU reference (torch autograd through
  tests/mol_torch.py, itself pinned to the oracle) to round-off;
* central finite differences of a functional (mass in a sphere at the final
  time) agree with it;
* the torch.autograd.Function wrapper returns the same gradient.
"""
import numpy as np
import pytest

from camr_b200 import hydro, native
from camr_b200 import problems as P

pytestmark = pytest.mark.gpu


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _adj():
    from camr_b200 import adjoint
    return adjoint


def init_state(n, seed):
    import oracle
    lev = oracle.make_level(n)
    p = oracle.default_params(do_mol=1, cfl=0.3)
    s = P.random_smooth(n, seed=seed)
    oracle.init_finalize("restate", p, lev, s)
    return s


def blast(n, p_blast=20.0, r=0.1):
    """rho = 1 + 0.05 sin(2 pi x) cos(2 pi y) sin(2 pi z), p = 1, a centred
    blast p = p_blast for r < r; zero velocity (initData epilogue applied)."""
    x, y, z = P.cell_centres(n, dx=tuple(1.0 / v for v in n))
    X, Y, Z = x[None, None, :], y[None, :, None], z[:, None, None]
    rho = 1.0 + 0.05 * np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y) * np.sin(2 * np.pi * Z)
    rho = np.broadcast_to(rho, (n[2], n[1], n[0])).copy()
    rr = np.sqrt((X - 0.5) ** 2 + (Y - 0.5) ** 2 + (Z - 0.5) ** 2)
    p = np.where(rr < r, p_blast, 1.0) * np.ones_like(rho)
    s = np.zeros((P.NVAR,) + rho.shape)
    s[P.URHO] = rho
    s[P.UEINT] = p / 0.4
    s[P.UEDEN] = s[P.UEINT]
    s[P.UTEMP] = 0.4 * (s[P.UEINT] / rho) * 26.93 / 8.31446261815324e7
    s[P.UFS] = rho
    return s, rr


def test_adjoint_forward_matches_level():
    torch = _torch()
    adjoint = _adj()
    n = (16, 12, 10)
    s = init_state(n, 3)
    geom = hydro.make_geom(n)
    prm = native.default_params(do_mol=1, cfl=0.3)
    L = hydro.Level(geom, prm, use_graph=False)
    L.set_state(s)
    dts = []
    for _ in range(4):
        L.advance(1)
        dts.append(L.last_dt())
    ref = L.get_state()
    L.close()
    A = adjoint.AdjointLevel(geom, prm, checkpoint_every=2)
    out = A.forward(torch.from_numpy(s).cuda(), 4)
    torch.cuda.synchronize()
    assert np.array_equal(A.dts(), np.array(dts))
    assert np.array_equal(out.cpu().numpy(), ref)
    A.close()


def test_adjoint_matches_taped_reference():
    torch = _torch()
    adjoint = _adj()
    import mol_torch as MT
    n = (12, 10, 8)
    s = init_state(n, 7)
    geom = hydro.make_geom(n)
    prm = native.default_params(do_mol=1, cfl=0.3)
    A = adjoint.AdjointLevel(geom, prm, checkpoint_every=2)
    A.forward(torch.from_numpy(s).cuda(), 3)
    dts = A.dts()
    rng = np.random.default_rng(11)
    lam = rng.standard_normal(s.shape)
    lam[P.UTEMP] = 0.0
    g = A.backward(torch.from_numpy(lam).cuda()).cpu().numpy()
    assert A.error()[0] == 0
    A.close()
    S0 = torch.from_numpy(s.copy()).requires_grad_(True)
    S = S0
    dx = tuple(geom.dx[d] for d in range(3))
    for dt in dts:
        S = MT.step(S, float(dt), dx, MT.Par())
    (S * torch.from_numpy(lam)).sum().backward()
    ref = S0.grad.numpy()
    for c in range(P.NVAR):
        if c == P.UTEMP:
            continue
        err = np.linalg.norm(g[c] - ref[c]) / max(np.linalg.norm(ref[c]), 1e-300)
        assert err < 1e-9, (c, err)


def test_adjoint_finite_differences():
    torch = _torch()
    adjoint = _adj()
    n = (24, 24, 24)
    s, rr = blast(n)
    geom = hydro.make_geom(n)
    prm = native.default_params(do_mol=1, cfl=0.3)
    A = adjoint.AdjointLevel(geom, prm, checkpoint_every=3)
    nsteps = 8
    dV = 1.0 / (n[0] * n[1] * n[2])
    mask = (rr < 0.2).astype(np.float64) * np.ones((n[2], n[1], n[0]))
    out = A.forward(torch.from_numpy(s).cuda(), nsteps)
    dts = A.dts()
    lam = np.zeros_like(s)
    lam[P.URHO] = mask * dV
    g = A.backward(torch.from_numpy(lam).cuda()).cpu().numpy()
    # perturb the initial density at fixed p, u: URHO and the first species
    grad_rho = g[P.URHO] + g[P.UFS]

    def J(state):
        o = A.forward(torch.from_numpy(state).cuda(), nsteps, fixed_dts=dts).cpu().numpy()
        return (o[P.URHO] * mask).sum() * dV

    rng = np.random.default_rng(64)
    cells = [(12, 12, 12), (12, 13, 14), (10, 12, 12)]
    cells += [tuple(int(v) for v in rng.integers(6, 18, size=3)) for _ in range(5)]
    for (k, j, i) in cells:
        eps = 1e-6 * s[P.URHO, k, j, i]
        sp, sm = s.copy(), s.copy()
        for st, sg in ((sp, 1.0), (sm, -1.0)):
            st[P.URHO, k, j, i] += sg * eps
            st[P.UFS, k, j, i] += sg * eps
        fd = (J(sp) - J(sm)) / (2 * eps)
        ad = grad_rho[k, j, i]
        assert abs(fd - ad) <= 1e-5 * max(abs(fd), abs(ad)) + 1e-14, ((k, j, i), fd, ad)
    A.close()
    del out


def test_autograd_function_gives_library_gradient():
    torch = _torch()
    adjoint = _adj()
    n = (12, 12, 12)
    s = init_state(n, 9)
    geom = hydro.make_geom(n)
    prm = native.default_params(do_mol=1, cfl=0.3)
    A = adjoint.AdjointLevel(geom, prm, checkpoint_every=2)
    S0 = torch.from_numpy(s).cuda().requires_grad_(True)
    S = adjoint.mol_steps(S0, A, 3)
    w = torch.linspace(0.0, 1.0, S[0].numel(), dtype=torch.float64, device="cuda")
    J = (S[P.URHO].reshape(-1) * w).sum()
    J.backward()
    lam = torch.zeros_like(S)
    lam[P.URHO] = w.reshape(S[0].shape)
    ref = A.backward(lam)
    assert torch.equal(S0.grad, ref)
    A.close()
