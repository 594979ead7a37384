"""rb_div_g (include/rb_detmath.h) equals the IEEE division x / 9.81f it replaces.

The HLLC kernel forms the star-depth estimate hs * hs / g with a multiply and a
fused multiply-add (division by a known constant, Brisebarre-Muller-Raina); the
CPU oracle keeps the division. This compiles a small C program against the header
and compares the two bit for bit on every non-negative float, from +0 through the
subnormals to +inf, plus negative values and NaN, with the oracle's compiler
settings (no contraction; the fused operation is the explicit fmaf).
"""

from __future__ import annotations

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include "rb_detmath.h"

static float bits(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static uint32_t word(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

int main(void) {
  long long bad = 0, tried = 0;
  /* every float with the sign bit clear: +0, subnormals, normals, +inf, and the NaNs */
#pragma omp parallel for reduction(+ : bad, tried) schedule(static)
  for (long long u = 0; u <= 0x7fffffffLL; u++) {
    const float x = bits((uint32_t)u);
    volatile float q = x / 9.81f;
    const float got = rb_div_g(x);
    tried++;
    if (x != x) { bad += got == got; continue; }  /* NaN in, NaN out */
    bad += word(got) != word(q);
  }
  /* negative values (a sign-flipped sample of every exponent) */
  for (uint32_t e = 0; e < 256; e++)
    for (uint32_t m = 0; m < (1u << 23); m += 4099) {
      const float x = bits(0x80000000u | (e << 23) | m);
      volatile float q = x / 9.81f;
      const float got = rb_div_g(x);
      tried++;
      if (x != x) bad += got == got;
      else bad += word(got) != word(q);
    }
  printf("tried %lld mismatches %lld\n", tried, bad);
  return bad != 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_div_g_is_the_ieee_quotient_for_every_float(tmp_path):
    src = tmp_path / "d.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "d"
    subprocess.run(["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", str(exe), "-lm"], check=True)  # fmt: skip
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout
    assert "mismatches 0" in out.stdout
