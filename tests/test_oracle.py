"""The CPU oracle pinned against golden vectors produced by the reference
itself (tests/golden/make_golden.py) and against the reference's own
known-answer tests.  No GPU needed."""
import gzip
import hashlib
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_json
from mersenne_trinomial_b200 import workloads as W


def sha(b):
    return hashlib.sha256(b).hexdigest()


def words_of(hexlist):
    return np.array([int(h, 16) for h in hexlist], dtype=np.uint64)


# ------------------------------------------------------------------- sieve
@pytest.mark.parametrize("idx", [0, 1, 2])
def test_sieve_config1_matches_sieve_ref(oracle, idx):
    case = load_json("sieve.json")["cases"][idx]
    best = oracle.sieve(case["r"], case["depth"], case["smax"])
    got = "".join(l + "\n" for l in oracle.cert_lines(best))
    with gzip.open(os.path.join(GOLDEN, case["file"]), "rt") as f:
        want = f.read()
    assert got == want
    assert sha(got.encode()) == case["sha256"]


@pytest.mark.parametrize("r,depth,smax", [(136279841, 11, 30000), (74207281, 10, 20000),
                                           (101, 9, 100), (136279841, 20, 999999)])
def test_sieve_reference_selftest_configs(oracle, r, depth, smax):
    case = [c for c in load_json("sieve.json")["cases"]
            if (c["r"], c["depth"], c["smax"]) == (r, depth, smax)][0]
    best = oracle.sieve(r, depth, smax)
    txt = "".join(l + "\n" for l in oracle.cert_lines(best))
    assert txt.count("\n") == case["lines"]
    assert sha(txt.encode()) == case["sha256"]


@pytest.mark.parametrize("r,depth,smax", [(101, 9, 100), (136279841, 11, 3000),
                                           (74207281, 10, 2000), (44687, 9, 5000)])
def test_sieve_vs_brute_force(oracle, r, depth, smax):
    """sieve_ref.cpp:142-160 oracle: enumerate irreducibles, evaluate directly."""
    assert (oracle.sieve(r, depth, smax) == oracle.sieve_brute(r, depth, smax)).all()


def test_sieve_known_answer(oracle):
    # README example line '33 5 p29' at r = 136279841
    best = oracle.sieve(136279841, 8, 40)
    assert oracle.cert_lines(best)[[l.split()[0] for l in oracle.cert_lines(best)].index("33")] == "33 5 p29"


def test_sieve_rejects_bad_r(oracle):
    with pytest.raises(ValueError):
        oracle.sieve(127, 7, 50)          # 127 = 2^7 - 1


# ----------------------------------------------------------------- squaring
def test_square_fixtures(oracle):
    for c in load_json("square.json")["cases"]:
        if c["k"] >= 256:
            continue
        got = oracle.trin_square_k(oracle.x_state(c["r"]), c["r"], c["s"], c["k"])
        assert sha(got.tobytes()) == c["sha256"], c
        if "words" in c:
            assert (got == words_of(c["words"])).all()


@pytest.mark.slow
def test_square_config2_fixtures(oracle):
    for c in load_json("square.json")["cases"]:
        if c["k"] != 4096:
            continue
        got = oracle.trin_square_k(oracle.x_state(c["r"]), c["r"], c["s"], c["k"])
        assert sha(got.tobytes()) == c["sha256"]


@pytest.mark.slow
def test_square_benchmark_workload_fixtures(oracle):
    """F_256 at r = 136279841 for the benchmark's first two s values, as the
    reference's kernels computed it (about 30 s of oracle time each)."""
    cases = [c for c in load_json("square.json")["cases"] if c["k"] == 256]
    assert len(cases) == 2
    for c in cases:
        got = oracle.trin_square_k(oracle.x_state(c["r"]), c["r"], c["s"], c["k"])
        assert sha(got.tobytes()) == c["sha256"], c["s"]


def test_frobenius_kat(oracle):
    # r = 31, s = 3: x^31 + x^3 + 1 is primitive, so F_31 = x (trinomial_stage2.cu:75-99)
    assert list(oracle.trin_square_k(oracle.x_state(31), 31, 3, 31)) == [2]


def test_square_vs_naive(oracle):
    rng = np.random.default_rng(5)
    for r, s in [(4423, 1200), (127, 1), (127, 63), (193, 64), (1031, 500)]:
        st = rng.integers(0, 2**63, size=oracle.words(r), dtype=np.uint64)
        if r & 63:
            st[-1] &= np.uint64((1 << (r & 63)) - 1)
        a = oracle.trin_square_k(st, r, s, 3)
        b = st
        for _ in range(3):
            b = oracle.trin_square_naive(b, r, s)
        assert (a == b).all()


def test_interval_product_fixture(oracle):
    p = load_json("square.json")["products"][0]
    r, s = p["r"], p["s"]
    F = oracle.x_state(r)
    acc = np.zeros(oracle.words(r), dtype=np.uint64)
    acc[0] = 1
    for k in range(1, p["k1"] + 1):
        F = oracle.trin_square_k(F, r, s, 1)
        if k >= p["k0"]:
            t = F.copy()
            t[0] ^= np.uint64(2)
            prod = oracle.comb_mul(acc, r, t, r)
            acc = oracle.mod_trinomial(prod, 2 * r - 1, r, s)
    assert (acc == words_of(p["words"])).all()


# ------------------------------------------------------------------- FFT
def test_cantor_basis_fixture(oracle):
    fx = load_json("fft.json")
    assert [format(int(x), "x") for x in oracle.cantor_basis()] == fx["basis"]
    W10 = oracle.fft_twiddles(10)
    assert sha(W10.tobytes()) == fx["twiddles_m10_sha256"]


def test_fft_transform_fixtures(oracle):
    for t in load_json("fft.json")["transforms"]:
        f = W.splitmix64(t["seed"], 1 << t["m"])
        g = oracle.fft_fwd(f, t["m"])
        assert sha(g.tobytes()) == t["fwd_sha256"], t["m"]
        assert (oracle.fft_inv(g, t["m"]) == f).all()


def test_fft_product_fixtures(oracle):
    for c in load_json("fft.json")["products"]:
        if c["abits"] + c["bbits"] > 4_000_000:
            continue
        a = W.random_bits(c["abits"], c["seed_a"])
        b = W.random_bits(c["bbits"], c["seed_b"])
        out = oracle.fft_mul(a, c["abits"], b, c["bbits"])
        assert sha(out.tobytes()) == c["sha256"], c
        if c["abits"] * c["bbits"] <= 10**10:
            assert (out == oracle.comb_mul(a, c["abits"], b, c["bbits"])).all()


def test_gf64_mul_paths(oracle):
    rng = np.random.default_rng(3)
    for a, b in rng.integers(0, 2**63, size=(2000, 2), dtype=np.uint64):
        a, b = int(a) * 2 + 1, int(b)
        assert oracle.lib().orc_gf64_mul(a, b) == oracle.lib().orc_gf64_mul_bitref(a, b)


# ------------------------------------------------------------ verification
def test_factor_divides_matches_reference_verifier(oracle):
    for c in load_json("verify.json"):
        s, d, p = c["line"].split()
        got = oracle.factor_divides(c["r"], int(s), int(d), p[1:]) == 1
        assert got == c["divides"], c


def test_deep_kat(oracle):
    # the r = 136279841, s = 474 degree-41 factor (tsfactor_handoff.md:337)
    assert oracle.factor_divides(136279841, 474, 41, "3991ef16129") == 1
    assert oracle.factor_divides(136279841, 475, 41, "3991ef16129") == 0
    assert oracle.factor_divides(136279841, 474, 40, "3991ef16129") == -1


# -------------------------------------------------------------------- scan
def test_scan_oracle_matches_reference(oracle):
    fx = load_json("scan.json")
    r, k0, maxd = fx["r"], fx["k0"], fx["maxd"]
    best = oracle.sieve(r, k0, 350)
    surv = [s for s in range(2, 351) if int(best[s]) == 0xFFFFFFFFFFFFFFFF]
    assert surv == fx["survivors"]
    want = {int(l.split()[0]): l for l in fx["results"]}
    nfound = nu = nties = 0
    for s in surv:
        st, d, gdeg, g, mask = oracle.scan_one(r, s, k0, maxd)
        w = want[s].split()
        if st == 2:
            nu += 1
            assert w[1] == "u"
            continue
        assert st == 1
        nfound += 1
        nties += gdeg != d
        assert int(w[1]) == d
        if w[2].startswith("p"):
            assert mask == w[2][1:]
        else:
            # the reference without NTL defers the tie-break ('g<file>') for
            # d > 22; with a single factor (deg g == d) the factor is g itself
            assert w[2].startswith("g") and d > 22
            assert mask is None or (gdeg == d and mask == g)
    assert (len(surv), nfound, nu, nties) == (104, 102, 2, 3)   # trinomial_scan --selftest
