"""rb_quotient_nonneg (include/rb_detmath.h) equals the IEEE comparison it replaces.

The HLLC kernel reads the contact-wave speed only through ``s_star >= 0``; the
helper decides that comparison from the operands' signs and forms the quotient
only when a negative quotient could underflow to -0. This compiles a small C
program against the header and checks it against ``n / d >= 0.0f`` on every
combination of special values and on tens of millions of random and near-underflow
operand pairs, with the same compiler settings as the oracle (no contraction).
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

static uint64_t s = 0x9E3779B97F4A7C15ull;
static uint32_t next(void) { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return (uint32_t)(s >> 16); }
static float bits(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static long long bad = 0, tried = 0;
static void check(float n, float d) {
  if (d != d || !(fabsf(d) > 1.0e-12f)) return;
  volatile float q = n / d;
  int want = q >= 0.0f;
  tried++;
  if (rb_quotient_nonneg(n, d) != want) {
    if (bad < 10) printf("mismatch n=%a d=%a\n", n, d);
    bad++;
  }
}
int main(void) {
  const float sp[] = {0.0f, -0.0f, 1e-45f, -1e-45f, 1e-40f, -1e-40f, 1.17549435e-38f, -1.17549435e-38f, 1e-30f,
                      -1e-30f, 1e-12f, 1.1e-12f, -1.1e-12f, 1.0f, -1.0f, 3.0e38f, -3.0e38f, INFINITY, -INFINITY, NAN};
  const int ns = sizeof sp / sizeof sp[0];
  for (int i = 0; i < ns; i++)
    for (int j = 0; j < ns; j++) check(sp[i], sp[j]);
  for (long k = 0; k < 20000000; k++) check(bits(next()), bits(next()));
  for (long k = 0; k < 20000000; k++) {  /* near underflow: tiny n, large d */
    const float n = bits(next() & 0x807FFFFFu | ((next() % 40u) << 23));
    const float d = bits(next() & 0x807FFFFFu | ((100u + next() % 155u) << 23));
    check(n, d);
  }
  printf("tried %lld mismatches %lld\n", tried, bad);
  return bad != 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_quotient_sign_matches_ieee_division(tmp_path):
    src = tmp_path / "q.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "q"
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", str(exe), "-lm"], check=True)  # fmt: skip
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout
    assert "mismatches 0" in out.stdout
