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


def smooth_state(n, seed):
    """A smooth periodic flow with non-zero velocities (no kinks of the
    limiters or Riemann branches at the finite-difference scale)."""
    rng = np.random.default_rng(seed)
    x, y, z = P.cell_centres(n, dx=tuple(1.0 / v for v in n))
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    X, Y, Z = X.transpose(2, 1, 0), Y.transpose(2, 1, 0), Z.transpose(2, 1, 0)

    def f(a):
        ph = rng.uniform(0, 2 * np.pi, 3)
        k = rng.integers(1, 3, 3)
        return a * np.sin(2 * np.pi * k[0] * X + ph[0]) * np.sin(2 * np.pi * k[1] * Y + ph[1]) \
            * np.sin(2 * np.pi * k[2] * Z + ph[2])

    rho = 1.0 + f(0.2)
    u = [0.3 + f(0.2), -0.2 + f(0.2), 0.1 + f(0.2)]
    p = 1.0 + f(0.3)
    s = np.zeros((P.NVAR,) + rho.shape)
    s[P.URHO] = rho
    for d in range(3):
        s[P.UMX + d] = rho * u[d]
    s[P.UEINT] = p / 0.4
    s[P.UEDEN] = s[P.UEINT] + 0.5 * rho * (u[0] ** 2 + u[1] ** 2 + u[2] ** 2)
    s[P.UTEMP] = 0.4 * (s[P.UEINT] / rho) * 26.93 / 8.31446261815324e7
    s[P.UFS] = rho
    return s


def test_adjoint_finite_differences():
    """d/d rho0 of the mass inside a sphere after 8 steps, perturbing the
    initial density at fixed pressure and velocity (URHO, the first species
    and the momenta / energies that carry u and p)."""
    torch = _torch()
    adjoint = _adj()
    n = (24, 24, 24)
    s = smooth_state(n, 5)
    x, y, z = P.cell_centres(n, dx=tuple(1.0 / v for v in n))
    rr = np.sqrt((x[None, None, :] - 0.5) ** 2 + (y[None, :, None] - 0.5) ** 2 +
                 (z[:, None, None] - 0.5) ** 2)
    geom = hydro.make_geom(n)
    prm = native.default_params(do_mol=1, cfl=0.3)
    A = adjoint.AdjointLevel(geom, prm, checkpoint_every=3)
    nsteps = 8
    dV = 1.0 / (n[0] * n[1] * n[2])
    mask = (rr < 0.2).astype(np.float64)
    A.forward(torch.from_numpy(s).cuda(), nsteps)
    dts = A.dts()
    lam = np.zeros_like(s)
    lam[P.URHO] = mask * dV
    g = A.backward(torch.from_numpy(lam).cuda()).cpu().numpy()
    rho = s[P.URHO]
    u = s[P.UMX:P.UMZ + 1] / rho
    ke = 0.5 * (u ** 2).sum(axis=0)
    # d(state)/d(rho) at fixed p, u
    grad_rho = g[P.URHO] + g[P.UFS] + (g[P.UMX:P.UMZ + 1] * u).sum(axis=0) + g[P.UEDEN] * ke

    def J(state):
        o = A.forward(torch.from_numpy(state).cuda(), nsteps, fixed_dts=dts).cpu().numpy()
        return (o[P.URHO] * mask).sum() * dV

    # cells inside the sphere, where dJ/drho is of order dV (far outside it
    # the gradient is below the finite differences' round-off floor)
    rng = np.random.default_rng(64)
    inside = np.argwhere(mask > 0)
    cells = [tuple(int(v) for v in inside[t]) for t in rng.choice(len(inside), 8, replace=False)]
    errs = []
    for (k, j, i) in cells:
        eps = 1e-6 * rho[k, j, i]
        res = []
        for sg in (1.0, -1.0):
            st = s.copy()
            r1 = rho[k, j, i] + sg * eps
            st[P.URHO, k, j, i] = r1
            st[P.UFS, k, j, i] = r1
            st[P.UMX:P.UMZ + 1, k, j, i] = r1 * u[:, k, j, i]
            st[P.UEDEN, k, j, i] = s[P.UEINT, k, j, i] + r1 * ke[k, j, i]
            res.append(J(st))
        fd = (res[0] - res[1]) / (2 * eps)
        ad = grad_rho[k, j, i]
        errs.append(abs(fd - ad) / max(abs(fd), abs(ad)))
    A.close()
    assert np.median(errs) <= 1e-6, errs
    assert max(errs) <= 1e-5, errs


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
    # the scatter sums use FP64 atomics: two runs agree to round-off
    assert torch.allclose(S0.grad, ref, rtol=1e-12, atol=1e-14 * float(ref.abs().max()))
    A.close()
