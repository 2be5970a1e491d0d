"""The taped torch restatement of the MOL step (tests/mol_torch.py) against
the oracle on the CPU: same inputs, same dt sequence, relative difference at
round-off level.  This pins the reference gradient the adjoint tests use."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
from camr_b200 import problems as P  # noqa: E402

import mol_torch as MT  # noqa: E402


def test_mol_torch_step_matches_oracle(oracle_kind):
    n = (12, 10, 8)
    lev = oracle.make_level(n)
    p = oracle.default_params(do_mol=1, cfl=0.3)
    s = P.random_smooth(n, seed=5)
    oracle.init_finalize(oracle_kind, p, lev, s)
    dt = 0.5 * oracle.est_dt(oracle_kind, p, lev, s)
    dts = [dt, 0.9 * dt, 1.1 * dt]
    ref = s.copy()
    oracle.advance_fixed_dt(oracle_kind, p, lev, ref, dts)
    S = torch.from_numpy(s.copy())
    dx = tuple(lev.dx[d] for d in range(3))
    Pt = MT.Par()
    for dtv in dts:
        S = MT.step(S, dtv, dx, Pt)
    got = S.numpy()
    for c in (0, 1, 2, 3, 4, 5, 7, 8, 9):
        rel = np.abs(got[c] - ref[c]).max() / np.abs(ref[c]).max()
        assert rel < 1e-12, (c, rel)
