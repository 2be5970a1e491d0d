"""The multiply-shift division of the kernels' flat-index decoding
(FastDiv / decode3 in camr_b200/csrc/fastdiv.h) equals integer
division: the header's host path is compiled with g++ and checked against
`/` for every divisor up to 5000 and sampled larger ones, on dividends at
and around every multiple boundary and at random up to 2^31 - 1, and the
decoded (i, j, k) of sampled region shapes against the 64-bit formula."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "camr_b200", "csrc")

PROGRAM = r"""
#include <cstdio>
#include <random>
#include <vector>
#include "fastdiv.h"
using namespace camr;
static long bad = 0;
static void check(unsigned n, unsigned d, const FastDiv& f) {
  if (fastdiv(n, f) != n / d) {
    if (bad < 5) std::printf("n=%u d=%u got %u want %u\n", n, d, fastdiv(n, f), n / d);
    ++bad;
  }
}
int main() {
  std::mt19937_64 rng(12345);
  const unsigned top = 0x7fffffffu;
  std::vector<unsigned> divs;
  for (unsigned d = 1; d <= 5000; ++d) divs.push_back(d);
  for (int b = 13; b <= 30; ++b) {
    divs.push_back((1u << b) - 1);
    divs.push_back(1u << b);
    divs.push_back((1u << b) + 1);
  }
  for (int r = 0; r < 2000; ++r) divs.push_back(1u + unsigned(rng() % top));
  for (unsigned d : divs) {
    const FastDiv f = make_fastdiv(d);
    for (unsigned n = 0; n < 64; ++n) check(n, d, f);
    check(top, d, f);
    check(top - 1, d, f);
    for (int r = 0; r < 200; ++r) {
      const unsigned q = unsigned(rng() % (top / d + 1));
      const unsigned long long m = (unsigned long long)q * d;
      for (long long e = -1; e <= 1; ++e) {
        const long long n = (long long)m + e;
        if (n >= 0 && n <= (long long)top) check(unsigned(n), d, f);
      }
      check(unsigned(rng() % (unsigned long long)(top + 1ull)), d, f);
    }
  }
  // region decoding against the 64-bit formula
  for (int r = 0; r < 3000; ++r) {
    const int n0 = 1 + int(rng() % 700), n1 = 1 + int(rng() % 700);
    const long long cap = ((1ll << 31) - 1) / ((long long)n0 * n1);
    const int n2 = 1 + int(rng() % (unsigned long long)(cap < 700 ? cap : 700));
    const Decode3 c = make_decode3(n0, n1, n2);
    if (!c.fast) { ++bad; continue; }
    const long long cnt = (long long)n0 * n1 * n2;
    for (int s = 0; s < 100; ++s) {
      const long long t = (s == 0) ? cnt - 1 : (long long)(rng() % (unsigned long long)cnt);
      int i, j, k;
      decode3(c, t, i, j, k);
      const long long nxy = (long long)n0 * n1;
      const int kk = int(t / nxy);
      const long long rem = t - kk * nxy;
      const int jj = int(rem / n0), ii = int(rem - (long long)jj * n0);
      if (i != ii || j != jj || k != kk) ++bad;
    }
  }
  if (make_decode3(2048, 1024, 1024).fast) ++bad;  // 2^31 cells: the 64-bit path
  std::printf("bad=%ld\n", bad);
  return bad != 0;
}
"""


def test_fastdiv_equals_integer_division(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    src = tmp_path / "fd.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "fd"
    subprocess.run([gxx, "-O2", "-std=c++17", "-I", CSRC, str(src),
                    "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout
    assert "bad=0" in out.stdout
