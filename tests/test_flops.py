"""The algorithmic flop counts bench.py reports (FLOPS_PER_ZONE_UPDATE) are
recounted on the reference's own per-box hydro compiled with a counting
amrex::Real (oracle/count_flops.py).  CPU only."""
import os
import sys

import numpy as np
import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HAVE = os.path.exists(oracle.lib_path_flops()) and os.path.exists(oracle.lib_path("ref"))


@pytest.mark.skipif(not HAVE, reason="oracle/_ref not built (reference sources absent)")
@pytest.mark.parametrize("method", ["ctu_ppm", "mol_plm"])
def test_bench_flop_constants_match_the_counting_oracle(method):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, ROOT)
    import bench
    import count_flops
    got = count_flops.count(method)["per_zone_update"]["flops"]
    assert abs(bench.FLOPS_PER_ZONE_UPDATE[method] - got) <= 1e-3 * got, (method, got)
