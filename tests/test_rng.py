"""The Philox4x32-10 stream shared by the engine and the oracle hook
(include/mcb200_rng.h): published known-answer vectors of the generator
(Salmon et al., SC'11, Random123 distribution) and the uniform mapping."""
import os
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <stdio.h>
#include "mcb200_rng.h"
int main(void) {
  const uint32_t in[3][6] = {
    {0u, 0u, 0u, 0u, 0u, 0u},
    {0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu},
    {0x243f6a88u, 0x85a308d3u, 0x13198a2eu, 0x03707344u, 0xa4093822u, 0x299f31d0u}};
  for (int t = 0; t < 3; ++t) {
    mcb200_philox_block b = mcb200_philox4x32_10(in[t][0], in[t][1], in[t][2], in[t][3], in[t][4], in[t][5]);
    printf("%08x %08x %08x %08x\n", b.w[0], b.w[1], b.w[2], b.w[3]);
  }
  printf("%.17g %.17g\n", mcb200_bits_to_unit(0u, 0u), mcb200_bits_to_unit(0xffffffffu, 0xffffffffu));
  double lo = 1, hi = 0, sum = 0;
  for (uint32_t n = 0; n < 200000; ++n) {
    double u = mcb200_uniform(42ull, 7u, 3u, 0u, n);
    if (u < lo) lo = u;
    if (u > hi) hi = u;
    sum += u;
  }
  printf("%.17g %.17g %.17g\n", lo, hi, sum / 200000);
  return 0;
}
"""


@pytest.fixture(scope="module")
def output():
    with tempfile.TemporaryDirectory() as tmp:
        src = os.path.join(tmp, "kat.c")
        exe = os.path.join(tmp, "kat")
        with open(src, "w") as f:
            f.write(PROGRAM)
        subprocess.run(["gcc", "-O2", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        return subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")


def test_known_answers(output):
    assert output[0] == "6627e8d5 e169c58d bc57ac4c 9b00dbd8"
    assert output[1] == "408f276d 41c83b0e a20bc7c6 6d5451fd"
    assert output[2] == "d16cfe09 94fdcceb 5001e420 24126ea1"


def test_unit_interval(output):
    lo, hi = (float(v) for v in output[3].split())
    assert lo == 2.0 ** -53 and hi == 1.0 - 2.0 ** -53
    mn, mx, mean = (float(v) for v in output[4].split())
    assert 0.0 < mn < 1e-4 and 1 - 1e-4 < mx < 1.0
    assert abs(mean - 0.5) < 0.005
