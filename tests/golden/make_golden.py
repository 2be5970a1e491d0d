"""Generate the golden fixtures from the reference's own hydro kernels.

Run where the reference sources exist (it builds oracle/_ref from the
reference checkout's Source/ directory named by CAMR_REF_SRC):
    CAMR_REF_SRC=<reference checkout>/Source python tests/golden/make_golden.py
Each fixture stores its exact inputs (small arrays) and the SHA-256 of the
exact bytes the reference produced, plus summary sums for diagnostics.
The reference's repository holds no tests, golden data or fixtures of its
own; these are the pins for its hydro path.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from camr_b200 import problems as P  # noqa: E402

BOX_CASES = [
    ("box_ctu_ppm_walls", dict(do_mol=0, ppm_type=1), (8, 6, 5),
     dict(periodic=(0, 1, 0), bc_lo=(2, 0, 4), bc_hi=(2, 0, 5)), 31),
    ("box_ctu_plm_sym", dict(do_mol=0, ppm_type=0), (7, 6, 6),
     dict(periodic=(0, 0, 0), bc_lo=(3, 5, 2), bc_hi=(4, 2, 3)), 32),
    ("box_mol_periodic", dict(do_mol=1, cfl=0.3), (8, 7, 5),
     dict(periodic=(1, 1, 1), bc_lo=(0, 0, 0), bc_hi=(0, 0, 0)), 33),
]
LEVEL_CASES = [
    ("run_sod_ctu_plm", dict(do_mol=0, ppm_type=0, cfl=0.8), (16, 6, 6),
     dict(periodic=(0, 1, 1), bc_lo=(2, 0, 0), bc_hi=(2, 0, 0)), "sod", 6),
    ("run_blobs_ctu_ppm", dict(do_mol=0, ppm_type=1, cfl=0.7), (10, 10, 8),
     dict(periodic=(1, 1, 1), bc_lo=(0, 0, 0), bc_hi=(0, 0, 0)), "blobs", 4),
    ("run_mol_walls", dict(do_mol=1, cfl=0.3), (10, 8, 6),
     dict(periodic=(0, 1, 0), bc_lo=(3, 0, 4), bc_hi=(5, 0, 2)), "random", 4),
]


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


def initial(kind, n, seed):
    dx = tuple(1.0 / v for v in n)
    if kind == "sod":
        return P.sod(n, dx)
    if kind == "blobs":
        return P.blobs(n, dx, nblobs=3, seed=seed, r_min=0.15, r_max=0.3)
    return P.random_smooth(n, seed=seed)


def main():
    oracle.build(ref=True)
    index = {}
    for name, cfg, n, bcs, seed in BOX_CASES:
        p = oracle.default_params(**cfg)
        lev = oracle.make_level(n, **bcs)
        s = P.random_smooth(n, seed=seed)
        oracle.init_finalize("ref", p, lev, s)
        border = oracle.expand_state("ref", p, lev, s)
        dt = 0.5 * oracle.est_dt("ref", p, lev, s)
        lo, hi = [0, 0, 0], [n[0] - 1, n[1] - 1, n[2] - 1]
        dsdt, flx, nass = oracle.hydro_box("ref", p, lo, hi, lo, hi, list(lev.bc_lo),
                                           list(lev.bc_hi), border, [-4, -4, -4],
                                           list(lev.dx), dt)
        assert nass == 0
        np.savez_compressed(os.path.join(HERE, name + ".npz"), state=s)
        index[name] = {"kind": "box", "cfg": cfg, "n": n, "bcs": bcs, "dt": dt,
                       "sha256_dsdt_flux": digest(dsdt, *flx),
                       "sum_dsdt": [float(v) for v in dsdt.sum(axis=(1, 2, 3))]}
    for name, cfg, n, bcs, kind, nsteps in LEVEL_CASES:
        p = oracle.default_params(**cfg)
        lev = oracle.make_level(n, **bcs)
        s0 = initial(kind, n, 41)
        s = s0.copy()
        oracle.init_finalize("ref", p, lev, s)
        _, hist, nass = oracle.advance("ref", p, lev, s, nsteps)
        assert nass == 0
        np.savez_compressed(os.path.join(HERE, name + ".npz"), state=s0)
        index[name] = {"kind": "run", "cfg": cfg, "n": n, "bcs": bcs, "nsteps": nsteps,
                       "dt_hist": [float(v) for v in hist],
                       "sha256_state": digest(s),
                       "sum_state": [float(v) for v in s.sum(axis=(1, 2, 3))]}
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(index, f, indent=1)
    print("wrote", len(index), "fixtures")


if __name__ == "__main__":
    main()
