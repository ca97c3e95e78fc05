"""Division-free forms of correctly rounded float division used by the
deformation kernel, checked on the CPU against IEEE division.

The cubic B-spline weights (1-d)^3/6 and d^3/6 are formed on the device as
q0 = x * RN(1/6) followed by one fused multiply-add residual correction
(k_deform.cu, div6). Every step scales exactly with the binade of x while
the intermediates stay normal, so one full binade proves the identity for
all of them; the test runs two binades exhaustively (the unit binade and the
smallest one the weights reach, [2^-72, 2^-71)) plus random samples across
[2^-72, 1]. The same comparison over every positive float with a normal
quotient (2^31 values) also finds no difference.
"""
import os
import shutil
import subprocess

import pytest

SRC = r"""
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
static float f_of(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static uint32_t u_of(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static int div6_ok(float x) {
  const float r = 1.0f / 6.0f;
  const float q0 = x * r;
  const float e = fmaf(-q0, 6.0f, x);
  const float q1 = fmaf(e, r, q0);
  return u_of(q1) == u_of(x / 6.0f);
}
int main(void) {
  unsigned long bad = 0;
  const uint32_t lo[2] = {u_of(1.0f), u_of(ldexpf(1.0f, -72))};
  for (int b = 0; b < 2; ++b)
    for (uint32_t u = lo[b]; u < lo[b] + (1u << 23); ++u) bad += !div6_ok(f_of(u));
  uint64_t s = 0x9E3779B97F4A7C15ull;
  for (int k = 0; k < 4000000; ++k) {
    s ^= s << 13; s ^= s >> 7; s ^= s << 17;
    const float x = ldexpf(1.0f + (float)(s & 0x7fffff) / 8388608.0f, -(int)((s >> 23) % 73));
    bad += !div6_ok(x);
  }
  bad += !div6_ok(0.0f);
  printf("%lu\n", bad);
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_div6_matches_ieee_division(tmp_path):
    c = tmp_path / "div6.c"
    exe = tmp_path / "div6"
    c.write_text(SRC)
    # no contraction: the product and the two fused steps are explicit
    subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-o", str(exe), str(c), "-lm"])
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.strip()
    assert out == "0", f"{out} quotients differ from IEEE division"
    assert os.path.exists(exe)
