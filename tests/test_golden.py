"""The oracle restatement against the golden fixtures (CPU, no reference needed).

tests/golden/golden.json holds SHA-256 digests of the exact output bytes the
reference's own hydro kernels produced on the stored inputs
(tests/golden/make_golden.py); the restatement must reproduce them bit for
bit.  The same fixtures pin the GPU path in tests/test_gpu_parity.py.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
with open(os.path.join(HERE, "golden.json")) as f:
    GOLDEN = json.load(f)


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


def load_state(name):
    return np.load(os.path.join(HERE, name + ".npz"))["state"]


@pytest.fixture(scope="module", autouse=True)
def _built():
    if not os.path.exists(oracle.lib_path("restate")):
        oracle.build(ref=False)


@pytest.mark.parametrize("name", [k for k, v in GOLDEN.items() if v["kind"] == "box"])
def test_restatement_box_golden(name):
    g = GOLDEN[name]
    n = tuple(g["n"])
    p = oracle.default_params(**g["cfg"])
    lev = oracle.make_level(n, **{k: tuple(v) for k, v in g["bcs"].items()})
    s = load_state(name)
    border = oracle.expand_state("restate", p, lev, s)
    lo, hi = [0, 0, 0], [n[0] - 1, n[1] - 1, n[2] - 1]
    dsdt, flx, nass = oracle.hydro_box("restate", p, lo, hi, lo, hi, list(lev.bc_lo),
                                       list(lev.bc_hi), border, [-4, -4, -4], list(lev.dx),
                                       g["dt"])
    assert nass == 0
    assert digest(dsdt, *flx) == g["sha256_dsdt_flux"], dsdt.sum(axis=(1, 2, 3))


@pytest.mark.parametrize("name", [k for k, v in GOLDEN.items() if v["kind"] == "run"])
def test_restatement_run_golden(name):
    g = GOLDEN[name]
    n = tuple(g["n"])
    p = oracle.default_params(**g["cfg"])
    lev = oracle.make_level(n, **{k: tuple(v) for k, v in g["bcs"].items()})
    s = load_state(name).copy()
    oracle.init_finalize("restate", p, lev, s)
    _, hist, nass = oracle.advance("restate", p, lev, s, g["nsteps"])
    assert nass == 0
    assert [float(v) for v in hist] == g["dt_hist"]
    assert digest(s) == g["sha256_state"], s.sum(axis=(1, 2, 3))
