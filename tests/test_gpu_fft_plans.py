"""Both Taylor-stage plans of the Cantor transform give the reference's
transform: the x^2 + x cascade (the reference's own level order) and the
tau-level recursion (levels at x^(2^h) + x, streamed or in tile passes),
each forced with GF2E_FFT_TAYLOR on sizes where the default picks the
other, checked against the oracle's transform, the inverse and a product.
Plans are cached per process, so each plan runs in its own process."""
import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

SCRIPT = r"""
import sys
sys.path.insert(0, %(root)r)
import numpy as np
import mersenne_trinomial_b200 as M
from mersenne_trinomial_b200 import workloads as W
from oracle import oracle as O
for m in %(sizes)r:
    f = W.splitmix64(700 + m, 1 << m)
    F = M.CudaFFT()
    F.init(m)
    d = M.DeviceBuffer.from_array(f)
    F.fwd(d)
    assert (d.to_numpy(1 << m) == O.fft_fwd(f, m)).all(), ("fwd", m)
    F.inv(d)
    assert (d.to_numpy(1 << m) == f).all(), ("inv", m)
    F.fini()
for bits in %(prod_bits)r:
    a = W.random_bits(bits, 3)
    b = W.random_bits(bits + 77, 4)
    got = M.gf2x_fft_mul(a, bits, b, bits + 77)
    want = O.fft_mul(a, bits, b, bits + 77)
    assert (np.asarray(got)[: want.size] == want).all(), ("mul", bits)
print("ok")
"""


@pytest.mark.parametrize("plan,sizes,prod_bits", [
    ("tau", [3, 6, 9, 11, 13, 14], [5000, 200000]),
    ("cascade", [15, 16, 17, 19], [3_000_000]),
])
def test_forced_taylor_plan_matches_oracle(plan, sizes, prod_bits):
    env = dict(os.environ, GF2E_FFT_TAYLOR=plan)
    code = SCRIPT % {"root": ROOT, "sizes": sizes, "prod_bits": prod_bits}
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                         timeout=900)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip().endswith("ok")
