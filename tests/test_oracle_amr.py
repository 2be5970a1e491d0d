"""CPU tests of the oracle's two-level AMR driver (no GPU).

* conservation: on a periodic domain the total of every conserved
  component over the base level is constant to round-off across subcycled
  steps (reflux + average-down close the coarse-fine flux mismatch);
* one fine box covering the whole domain reproduces the single-level run on
  the fine grid bit for bit, and the base level equals its average-down;
* the restatement and the reference kernels agree bit for bit inside the
  two-level driver (skipped when oracle/_ref was not built).
"""
import os

import numpy as np
import pytest

import oracle
from camr_b200 import problems as P

HAVE_REF = os.path.exists(oracle.lib_path("ref"))

N0 = (16, 16, 16)
# two abutting boxes, one box crossing nothing, one at the periodic corner
BOXES = [((8, 8, 8), (15, 15, 23)), ((16, 8, 8), (23, 15, 15)),
         ((0, 24, 0), (7, 31, 7)), ((24, 0, 24), (31, 7, 31))]
METHODS = {
    "mol_plm": dict(do_mol=1, ppm_type=0, cfl=0.3),
    "ctu_ppm": dict(do_mol=0, ppm_type=1, cfl=0.5),
    "ctu_plm": dict(do_mol=0, ppm_type=0, cfl=0.5),
}


def box_array(boxes):
    return np.array([list(lo) + list(hi) for lo, hi in boxes], dtype=np.int32)


def fine_views(S1, boxes):
    out, off = [], 0
    for lo, hi in boxes:
        nb = [hi[d] - lo[d] + 1 for d in range(3)]
        size = P.NVAR * nb[0] * nb[1] * nb[2]
        out.append(S1[off:off + size].reshape(P.NVAR, nb[2], nb[1], nb[0]))
        off += size
    return out


@pytest.fixture(scope="module", autouse=True)
def _built():
    if not os.path.exists(oracle.lib_path("restate")):
        oracle.build(ref=False)


def run(kind, method, boxes, nsteps, **extra):
    p = oracle.default_params(**METHODS[method], **extra)
    lev = oracle.make_level(N0)
    S0, S1 = P.amr_initial(N0, boxes, nblobs=4, r_min=0.1, r_max=0.2)
    clock = np.zeros(4)
    bx = box_array(boxes)
    oracle.amr_run(kind, p, lev, bx, S0, S1, 0, do_init=True, clock=clock)
    start = S0.copy()
    hist, nerr = oracle.amr_run(kind, p, lev, bx, S0, S1, nsteps, first_step=True, clock=clock)
    assert nerr == 0
    return start, S0, S1, hist, clock


@pytest.mark.parametrize("method", list(METHODS))
def test_amr_conservation(method):
    start, S0, S1, hist, clock = run("restate", method, BOXES, 3)
    assert np.all(hist[:, 1] == hist[:, 0] / 2)
    assert clock[0] == pytest.approx(hist[:, 0].sum(), rel=1e-14)
    for comp in (P.URHO, P.UMX, P.UMY, P.UMZ, P.UEDEN):
        a, b = start[comp].sum(), S0[comp].sum()
        assert abs(a - b) <= 1e-13 * np.abs(start[comp]).sum(), comp
    # covered coarse cells hold the average of their fine cells
    for (lo, hi), F in zip(BOXES, fine_views(S1, BOXES)):
        c = F.reshape(P.NVAR, F.shape[1] // 2, 2, F.shape[2] // 2, 2, F.shape[3] // 2, 2)
        avg = 0.125 * c.sum(axis=(2, 4, 6))
        sub = S0[:, lo[2] // 2:hi[2] // 2 + 1, lo[1] // 2:hi[1] // 2 + 1, lo[0] // 2:hi[0] // 2 + 1]
        np.testing.assert_allclose(sub[:5], avg[:5], rtol=1e-14, atol=0)


@pytest.mark.parametrize("method", ["mol_plm", "ctu_ppm"])
def test_amr_full_cover_equals_single_level_fine(method):
    full = [((0, 0, 0), (2 * N0[0] - 1, 2 * N0[1] - 1, 2 * N0[2] - 1))]
    dt = 2e-3
    start, S0, S1, hist, _ = run("restate", method, full, 2, fixed_dt=dt)
    assert np.all(hist[:, 0] == dt) and np.all(hist[:, 1] == dt / 2)
    n1 = tuple(2 * v for v in N0)
    p = oracle.default_params(**METHODS[method], fixed_dt=dt)
    lev1 = oracle.make_level(n1)
    _, F0 = P.amr_initial(N0, full, nblobs=4, r_min=0.1, r_max=0.2)
    F0 = F0.reshape(P.NVAR, n1[2], n1[1], n1[0]).copy()
    oracle.init_finalize("restate", p, lev1, F0)
    oracle.advance_fixed_dt("restate", p, lev1, F0, [dt / 2] * 4)
    assert np.array_equal(S1.reshape(F0.shape), F0)


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built (reference sources absent)")
@pytest.mark.parametrize("method", list(METHODS))
def test_amr_restatement_equals_reference(method):
    a = run("restate", method, BOXES, 2)
    b = run("ref", method, BOXES, 2)
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
    assert np.array_equal(a[3], b[3])
