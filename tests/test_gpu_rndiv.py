"""The kernels' shared-reciprocal quotient (camr_b200/csrc/rndiv.h) equals
the device's IEEE division bit for bit on about 5 x 2^26 operand pairs
(camr_check_rn_div: random operands, quotients next to rounding midpoints,
integer ratios, special values)."""
import ctypes as C

import pytest

from camr_b200 import native

pytestmark = pytest.mark.gpu


def test_rn_div_matches_device_division():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    bad = C.c_int64(-1)
    for seed in (1, 2):
        native.check(native.lib().camr_check_rn_div(1 << 26, seed, C.byref(bad), None),
                     "camr_check_rn_div")
        assert bad.value == 0
