"""The division used by the FP64 species pass (``div_rn`` in
flash5_b200/csrc/hy_core.cuh): x / b from rb = RN(1 / b) with one FMA
correction (Markstein's theorem).  Restated here in C and compared bit for
bit with IEEE division on random operands (constants 3 and 6 of the PPM
formulas, runtime grid spacings, significands of all ones) and on the
special values that take the plain division.  The FP64 GPU parity tests
check the device function itself against the oracle's divisions."""
import os
import subprocess

import pytest

SRC = r"""
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
static uint64_t s = 0x243F6A8885A308D3ull;
static uint64_t nx(void) { s += 0x9E3779B97F4A7C15ull; uint64_t z = s;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull; z = (z ^ (z >> 27)) * 0x94D049BB133111EBull; return z ^ (z >> 31); }
static double rnd(int lo, int hi) { uint64_t m = nx() & 0xFFFFFFFFFFFFFull; int e = lo + (int)(nx() % (uint64_t)(hi - lo));
  uint64_t b = ((uint64_t)(e + 1023) << 52) | m; if (nx() & 1) b |= 1ull << 63; double d; memcpy(&d, &b, 8); return d; }
static double div_rn(double x, double b, double rb) {
  const double q0 = x * rb;
  const double a = fabs(q0), ax = fabs(x);
  if (a > 0x1p-960 && a < 0x1p1000 && ax > 0x1p-960 && ax < 0x1p1000) return fma(fma(-q0, b, x), rb, q0);
  return x / b;
}
static long bad = 0;
static void check(double x, double b) {
  double q = div_rn(x, b, 1. / b), r = x / b;
  if (memcmp(&q, &r, 8) && !(isnan(q) && isnan(r))) { if (bad < 5) printf("x=%a b=%a q=%a r=%a\n", x, b, q, r); ++bad; }
}
int main(void) {
  const double cs[] = {3., 6.};
  for (int c = 0; c < 2; ++c)
    for (long i = 0; i < 4000000; ++i) check(i % 7 ? rnd(-60, 60) : rnd(-1021, 1023), cs[c]);
  for (long i = 0; i < 8000000; ++i) {
    double b = rnd(-40, 40);
    if (i % 5 == 0) { uint64_t bb; memcpy(&bb, &b, 8); bb |= 0xFFFFFFFFFFFF0ull; memcpy(&b, &bb, 8); }
    check(rnd(-60, 60), b);
  }
  const double sp[] = {0., -0., 1e-310, -1e-310, 5e-324, 1e308, -1e308, INFINITY, -INFINITY, NAN};
  for (int i = 0; i < 10; ++i) { check(sp[i], 3.); check(sp[i], 6.); check(sp[i], 1e-3); check(sp[i], 7.5e9); }
  printf("mismatches %ld\n", bad);
  return bad != 0;
}
"""


def test_div_rn_equals_division(tmp_path):
    c = tmp_path / "div_rn.c"
    exe = tmp_path / "div_rn"
    c.write_text(SRC)
    try:
        subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-o", str(exe), str(c), "-lm"], check=True,
                       capture_output=True, text=True)
    except (OSError, subprocess.CalledProcessError) as e:
        pytest.skip(f"no C compiler: {e}")
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout
