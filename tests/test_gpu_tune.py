"""Autotuner on the GPU: every candidate verified against the default
configuration, and results under non-default tunings bit-exact vs the oracle."""
import numpy as np
import pytest

from conftest import load_json
from mersenne_trinomial_b200 import workloads as W

pytestmark = pytest.mark.gpu

TUNINGS = [
    dict(fft_tile_log=11, fft_cmin=2, fft_taylor_lv=1, fft_bfly_lv=1),
    dict(fft_tile_log=13, fft_cmin=16, fft_taylor_lv=2, fft_bfly_lv=2),
    dict(fft_tile_log=13, fft_cmin=4, fft_taylor_lv=3, fft_bfly_lv=1),
]


@pytest.fixture
def restore_tune(engine):
    from mersenne_trinomial_b200 import autotune as A
    saved = A.tune_get()
    yield A
    A.tune_set(**saved)


def test_fft_autotune_verifies_every_candidate(restore_tune):
    A = restore_tune
    res = A.fft_autotune(14, reps=1)
    assert len(res["candidates"]) == 3 * 4 * 3 * 3
    assert all(c["status"] == "ok" for c in res["candidates"])
    assert A.tune_get() == res["best"]
    assert res["best_fwd_inv_ms"] == pytest.approx(min(c["ms"] for c in res["candidates"]),
                                                   abs=1e-4)     # report prints 4 decimals


@pytest.mark.parametrize("tune", TUNINGS)
def test_transform_and_products_under_tuning(engine, oracle, restore_tune, tune):
    A = restore_tune
    A.tune_set(**tune)
    for m in (3, 9, 15, 18):
        f = W.splitmix64(700 + m, 1 << m)
        F = engine.CudaFFT()
        F.init(m)
        d = engine.DeviceBuffer.from_array(f)
        F.fwd(d)
        assert (d.to_numpy(1 << m) == oracle.fft_fwd(f, m)).all(), (tune, m)
        F.inv(d)
        assert (d.to_numpy(1 << m) == f).all(), (tune, m)
    for ab, bb in ((1, 1), (700, 5), (100000, 99999), (2**18 + 3, 2**17)):
        a, b = W.random_bits(ab, ab), W.random_bits(bb, bb + 1)
        want = oracle.comb_mul(a, ab, b, bb)
        got = engine.gf2x_fft_mul(a, ab, b, bb)
        assert (got[:len(want)] == want).all(), (tune, ab, bb)


def test_sieve_autotune_matches_fixture(engine, restore_tune):
    A = restore_tune
    case = load_json("sieve.json")["cases"][0]
    res = A.sieve_autotune(case["r"], case["depth"], case["smax"], reps=1)
    assert [c["sieve_strip_log"] for c in res["candidates"]] == [10, 11, 12, 13, 14]
    assert all(c["status"] in ("ok", "OVERFLOW") for c in res["candidates"])
    # the chosen strip width is now active and still reproduces the fixture
    import gzip, os
    from conftest import GOLDEN
    best = engine.run_sieve(case["r"], case["depth"], case["smax"])
    with gzip.open(os.path.join(GOLDEN, case["file"]), "rt") as f:
        assert "".join(l + "\n" for l in engine.cert_lines(best)) == f.read()
