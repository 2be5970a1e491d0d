"""rn_div (camr_b200/csrc/rndiv.h), the correctly rounded quotient from a
shared reciprocal with Markstein's fused multiply-add corrections, equals
the IEEE division bit for bit: the header's host path (std::fma, no FMA
contraction) is compiled with g++ and checked against `/` on random
operands over +-60 binades, on quotients placed next to rounding midpoints
(a = b * m for a midpoint m of two doubles, and its neighbours), on
integer ratios and on special operands (zeros, subnormals, huge values,
infinities, NaN).  The device path is the same operations (DMUL and DFMA
round to nearest like the host's); tests/test_gpu_rndiv.py checks it on
the GPU."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "camr_b200", "csrc")

PROGRAM = r"""
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstdint>
#include <random>
#include "rndiv.h"
using camr::rn_div;
static long bad = 0, n = 0;
static void chk(double a, double b) {
  volatile double vb = b;
  const double y = 1.0 / vb;
  const double q = rn_div(a, b, y);
  volatile double va = a;
  const double w = va / vb;
  uint64_t x1, x2;
  memcpy(&x1, &q, 8);
  memcpy(&x2, &w, 8);
  ++n;
  if (x1 != x2 && !(std::isnan(q) && std::isnan(w))) {
    if (bad < 5) std::printf("a=%a b=%a got %a want %a\n", a, b, q, w);
    ++bad;
  }
}
int main(int argc, char** argv) {
  const long N = argc > 1 ? atol(argv[1]) : 2000000;
  std::mt19937_64 rng(7);
  std::uniform_real_distribution<double> U(1.0, 2.0);
  auto sgn = [&]() { return (rng() & 1) ? 1.0 : -1.0; };
  for (long i = 0; i < N; ++i) {
    chk(sgn() * std::ldexp(U(rng), int(rng() % 121) - 60),
        sgn() * std::ldexp(U(rng), int(rng() % 121) - 60));
    // a / b next to the midpoint m between q and its successor
    const double q = std::ldexp(U(rng), int(rng() % 41) - 20);
    const double m = q + 0.5 * (std::nextafter(q, 1e300) - q);
    const double b = std::ldexp(double((rng() % 4096) * 2 + 1), int(rng() % 21) - 10);
    const double a = b * m;
    chk(a, b);
    chk(std::nextafter(a, 1e300), b);
    chk(std::nextafter(a, -1e300), b);
    chk(double(int64_t(rng() % 2000001) - 1000000), double(int64_t(rng() % 2001) - 1000));
  }
  const double sp[] = {0.0, -0.0, 1.0, -1.0, 3.0, 0.1, 1e-7, 1e-200, -1e-300, 1e300,
                       std::ldexp(1.0, -500), std::ldexp(1.0, 499), std::ldexp(1.0, 500),
                       std::ldexp(1.0, -501), 5e-324, INFINITY, -INFINITY, NAN};
  for (double a : sp)
    for (double b : sp) chk(a, b);
  std::printf("n=%ld bad=%ld\n", n, bad);
  return bad != 0;
}
"""


def test_rn_div_equals_ieee_division(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    src = tmp_path / "rd.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "rd"
    subprocess.run([gxx, "-O2", "-std=c++17", "-ffp-contract=off", "-I", CSRC, str(src), "-o",
                    str(exe)], check=True)
    out = subprocess.run([str(exe), "2000000"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout
    assert "bad=0" in out.stdout
