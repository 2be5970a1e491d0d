"""Algorithmic flops per zone-update of the hydro, counted on the reference's
own per-box code (test and measurement infrastructure).

oracle/_ref/libcamr_ref_flops.so is the reference's hydro_ctoprim,
hydro_srctoprim and hydro_umdrv compiled with amrex::Real = a counting double
(oracle/amrex_shim/camr_counted_real.H).  One 64^3 box (the box size of the
256^3 configuration) of each method's configuration data is run and its
additions, multiplications, divisions and square roots are counted (one flop
each; comparisons, abs and copysign are reported apart).  A CTU step runs
the hydro once per zone-update, an SSP-RK2 (MOL) step twice.

  python oracle/count_flops.py      # prints the counts as JSON

bench.py carries the resulting per-zone-update figures as constants;
tests/test_flops.py recounts them and checks the constants.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from camr_b200 import problems as P  # noqa: E402

# method -> (params, box size, initial data, hydro evaluations per step)
CASES = {
    "ctu_ppm": (dict(do_mol=0, ppm_type=1, cfl=0.7), 64, "blobs", 1),
    "ctu_plm": (dict(do_mol=0, ppm_type=0, cfl=0.8), 64, "blobs", 1),
    "mol_plm": (dict(do_mol=1, cfl=0.3), 64, "grf", 2),
}


def count(method):
    cfg, n, data, evals = CASES[method]
    N = 2 * n
    dx = (1.0 / N,) * 3
    if data == "blobs":
        s = P.blobs((N, N, N), dx, nblobs=16, seed=1)
    else:
        s, _ = P.grf_blast((N, N, N), seed=3)
    p = oracle.default_params(**cfg)
    lev = oracle.make_level((N, N, N))
    oracle.init_finalize("ref", p, lev, s)
    dt = oracle.est_dt("ref", p, lev, s)
    full = np.pad(s, ((0, 0), (4, 4), (4, 4), (4, 4)), mode="wrap")
    uin = np.ascontiguousarray(full[:, :n + 8, :n + 8, :n + 8])
    c = oracle.count_flops(p, (n, n, n), (0, 0, 0), (0, 0, 0), uin, dx, dt)
    per = {k: evals * v / n ** 3 for k, v in c.items()}
    return {"box": n, "hydro_per_step": evals, "per_zone_update": per}


if __name__ == "__main__":
    print(json.dumps({m: count(m) for m in CASES}, indent=1))
