"""The ESSE smoothing divides by the odd constants 3, 5, 7 with one
multiplication by the rounded reciprocal and one correction by the exact
residual (Markstein, IBM J. Res. Dev. 34(1), 1990):

    q0 = RN(x * RN(1/d));  r = fma(-q0, d, x);  q = fma(r, RN(1/d), q0)

The device helper is `div_const` in libirl_b200/csrc/cuda/k_esse.cu.  This
test runs the same three IEEE operations in C (fmaf) and compares them with
the correctly rounded x / d.  Away from the subnormal and overflow ranges the
sequence is invariant under scaling by powers of two, so one full binade
stands for all normal binades; the subnormal range, the smallest normal
binades and the largest ones are swept in full.
"""
from __future__ import annotations

import os
import subprocess

import pytest

SRC = r"""
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
static unsigned long long sweep(float d, uint32_t lo, uint32_t hi) {
  const float y = 1.0f / d;
  unsigned long long bad = 0;
  for (uint64_t u = lo; u <= hi; ++u) {
    for (int s = 0; s < 2; ++s) {
      uint32_t b = (uint32_t)u | (s ? 0x80000000u : 0u);
      float x;
      memcpy(&x, &b, 4);
      if (!isfinite(x) || b == 0x80000000u) continue;
      float q0 = x * y;
      float r = fmaf(-q0, d, x);
      float q = fmaf(r, y, q0);
      float w = x / d;
      if (memcmp(&q, &w, 4) != 0) ++bad;
    }
  }
  return bad;
}
int main(void) {
  const float ds[3] = {3.f, 5.f, 7.f};
  unsigned long long bad = 0;
  for (int k = 0; k < 3; ++k) {
    bad += sweep(ds[k], 0x00000000u, 0x01ffffffu);  /* subnormals, first normal binades */
    bad += sweep(ds[k], 0x3f800000u, 0x3fffffffu);  /* [1, 2) */
    bad += sweep(ds[k], 0x7e800000u, 0x7f7fffffu);  /* largest binades */
  }
  printf("%llu\n", bad);
  return 0;
}
"""


def test_markstein_division_by_odd_constants(tmp_path):
    c = tmp_path / "div.c"
    exe = tmp_path / "div"
    c.write_text(SRC)
    cc = os.environ.get("CC", "gcc")
    try:
        subprocess.run([cc, "-O2", "-march=native", "-ffp-contract=off", str(c), "-o", str(exe), "-lm"], check=True,
                       capture_output=True)
    except (OSError, subprocess.CalledProcessError) as e:  # pragma: no cover
        pytest.skip(f"no C compiler: {e}")
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    assert int(out.strip()) == 0
