"""Tuning knobs and the gcd-interval chooser: host logic only (no GPU)."""
import os
import subprocess
import sys

import pytest

from conftest import ROOT


def model_cost(k0, maxd, t_deg, t_gcd, L0, Lmax):
    """The expected-cost model restated: P(least degree > D) = k0 / D, one
    gcd at the end of every interval reached."""
    c, lo, L = 0.0, k0, L0
    while lo < maxd:
        hi = min(maxd, lo + L)
        c += (k0 / lo) * ((hi - lo) * t_deg + t_gcd)
        lo, L = hi, min(2 * L, Lmax)
    return c


def test_tune_defaults_and_validation(engine):
    from mersenne_trinomial_b200 import autotune as A
    d = A.tune_default()
    assert d == {"fft_tile_log": 0, "fft_cmin": 0, "fft_taylor_lv": 3, "fft_bfly_lv": 3,
                 "sieve_strip_log": 12}
    saved = A.tune_get()
    try:
        for bad in ({"fft_tile_log": 10}, {"fft_tile_log": 14}, {"fft_tile_log": -1},
                    {"fft_cmin": 3}, {"fft_cmin": -2},
                    {"fft_cmin": 32}, {"fft_taylor_lv": 0}, {"fft_taylor_lv": 4},
                    {"fft_bfly_lv": 4}, {"fft_bfly_lv": 0}, {"sieve_strip_log": 9},
                    {"sieve_strip_log": 15}):
            with pytest.raises(engine.Gf2eError):
                A.tune_set(**bad)
            assert A.tune_get() == saved          # a rejected set changes nothing
        got = A.tune_set(fft_tile_log=13, fft_cmin=16, fft_taylor_lv=1, fft_bfly_lv=1,
                         sieve_strip_log=14)
        assert got["fft_tile_log"] == 13 and got["sieve_strip_log"] == 14
        assert A.export_lines(got)[0] == "export GF2E_FFT_TILE_LOG=13"
    finally:
        A.tune_set(**saved)


def _tune_in_child(env_extra):
    env = dict(os.environ, **env_extra)
    code = ("import sys; sys.path.insert(0, %r); "
            "from mersenne_trinomial_b200 import autotune as A; print(A.tune_get())" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                         timeout=120)
    assert out.returncode == 0, out.stderr
    return eval(out.stdout.strip().splitlines()[-1]), out.stderr


def test_tune_environment_overrides(engine):
    got, _ = _tune_in_child({"GF2E_FFT_TILE_LOG": "11", "GF2E_FFT_BFLY_LV": "1",
                             "GF2E_SIEVE_STRIP_LOG": "13"})
    assert got["fft_tile_log"] == 11 and got["fft_bfly_lv"] == 1 and got["sieve_strip_log"] == 13
    got, err = _tune_in_child({"GF2E_FFT_TILE_LOG": "99"})
    assert got["fft_tile_log"] == 0 and "ignoring" in err


@pytest.mark.parametrize("k0,maxd,t_deg,t_gcd", [
    (24, 20000, 0.0185, 1.0), (24, 20000, 0.0185, 30.0), (5, 200, 1.0, 10.0),
    (24, 50000, 0.001, 0.0), (20, 4096, 2.0, 1e4)])
def test_choose_interval_is_model_optimum(engine, k0, maxd, t_deg, t_gcd):
    from mersenne_trinomial_b200 import autotune as A
    res = A.choose_interval(k0, maxd, t_deg, t_gcd)
    L0, Lmax = res["L0"], res["Lmax"]
    assert L0 & (L0 - 1) == 0 and Lmax & (Lmax - 1) == 0 and L0 <= Lmax
    assert res["expected_cost"] == pytest.approx(model_cost(k0, maxd, t_deg, t_gcd, L0, Lmax))
    # no schedule on the searched grid is cheaper
    best = min(model_cost(k0, maxd, t_deg, t_gcd, 1 << a, 1 << b)
               for a in range(0, 21) for b in range(a, 23))
    assert res["expected_cost"] <= best * (1 + 1e-9)


def test_choose_interval_monotone_in_gcd_cost(engine):
    from mersenne_trinomial_b200 import autotune as A
    prev = 0
    for t_gcd in (0.01, 0.1, 1.0, 10.0, 100.0, 1000.0):
        L0 = A.choose_interval(24, 20000, 0.02, t_gcd)["L0"]
        assert L0 >= prev
        prev = L0


def test_choose_interval_rejects_bad_arguments(engine):
    from mersenne_trinomial_b200 import autotune as A
    for args in ((0, 100, 1.0, 1.0), (24, 24, 1.0, 1.0), (24, 100, 0.0, 1.0),
                 (24, 100, 1.0, -1.0)):
        with pytest.raises(engine.Gf2eError):
            A.choose_interval(*args)


def test_choose_block_balances_squarings_and_modmuls(engine):
    from mersenne_trinomial_b200 import autotune as A
    assert A.choose_block(15e-3, 7.2e-6) == 46          # sqrt(2083) = 45.6
    assert A.choose_block(1.0, 1.0) == 2                 # floor
    assert A.choose_block(1.0, 1e-9) == 62               # cap
    for t_mul, t_sq in ((1e-2, 1e-5), (3e-3, 2e-5), (0.2, 1e-6)):
        m = A.choose_block(t_mul, t_sq)
        assert m % 2 == 0 and 2 <= m <= 62
        cost = lambda k: k * t_sq + t_mul / k
        assert cost(m) <= min(cost(k) for k in range(2, 63, 2)) * 1.05
    with pytest.raises(engine.Gf2eError):
        A.choose_block(0.0, 1.0)


def test_resolve_by_size_rule():
    from mersenne_trinomial_b200 import autotune as A
    d = {"fft_tile_log": 0, "fft_cmin": 0, "fft_taylor_lv": 3, "fft_bfly_lv": 2,
         "sieve_strip_log": 12}
    assert A.resolve_by_size(d, 16)["fft_tile_log"] == 11
    assert A.resolve_by_size(d, 20)["fft_tile_log"] == 12
    assert A.resolve_by_size(d, 24) == dict(d, fft_tile_log=13, fft_cmin=8)
    assert A.resolve_by_size(dict(d, fft_tile_log=12), 24)["fft_tile_log"] == 12
