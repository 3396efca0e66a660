"""Sieve progression lists that fill up: a progression that finds the strip
or heavy list full is marked inline by the thread that found it, so best[]
is unchanged.  The list capacities are lowered from the host
(GF2E_SIEVE_STRIP_CAP / GF2E_SIEVE_HEAVY_CAP, read at each call) until
nearly every progression spills, and the result is compared with the
oracle and with the reference's golden output."""
import gzip
import os

import pytest

from conftest import GOLDEN, load_json

pytestmark = pytest.mark.gpu


@pytest.fixture
def tiny_lists(monkeypatch):
    monkeypatch.setenv("GF2E_SIEVE_STRIP_CAP", "3")
    monkeypatch.setenv("GF2E_SIEVE_HEAVY_CAP", "2")


def test_spilled_lists_give_the_same_sieve(engine, oracle, tiny_lists):
    case = load_json("sieve.json")["cases"][0]
    best = engine.run_sieve(case["r"], case["depth"], case["smax"])
    got = "".join(l + "\n" for l in engine.cert_lines(best))
    with gzip.open(os.path.join(GOLDEN, case["file"]), "rt") as f:
        assert got == f.read()
    for r, depth, smax in [(136279841, 22, 200000), (4423, 14, 2211)]:
        assert (engine.run_sieve(r, depth, smax) == oracle.sieve(r, depth, smax)).all(), (r, depth)


def test_caps_are_read_at_each_call(engine, oracle, monkeypatch):
    r, depth, smax = 44687, 18, 22343
    want = oracle.sieve(r, depth, smax)
    for strip_cap, heavy_cap in [("1", "1"), ("100000000", "100000000"), ("64", "0")]:
        monkeypatch.setenv("GF2E_SIEVE_STRIP_CAP", strip_cap)
        monkeypatch.setenv("GF2E_SIEVE_HEAVY_CAP", heavy_cap)
        assert (engine.run_sieve(r, depth, smax) == want).all(), (strip_cap, heavy_cap)
