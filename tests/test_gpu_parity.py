"""CUDA engine vs the oracle and the reference's golden vectors, through the
C ABI (libgf2e.so).  Bit-exact everywhere: all arithmetic is over GF(2)."""
import gzip
import hashlib
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_json
from mersenne_trinomial_b200 import workloads as W

pytestmark = pytest.mark.gpu


def sha(b):
    return hashlib.sha256(b).hexdigest()


def words_of(hexlist):
    return np.array([int(h, 16) for h in hexlist], dtype=np.uint64)


def rand_state(rng, r):
    st = rng.integers(0, 2**63, size=(r + 63) // 64, dtype=np.uint64) * np.uint64(2) + \
        rng.integers(0, 2, size=(r + 63) // 64, dtype=np.uint64)
    if r & 63:
        st[-1] &= np.uint64((1 << (r & 63)) - 1)
    return st


# ------------------------------------------------------------------- sieve
@pytest.mark.parametrize("idx", [0, 1, 2])
def test_sieve_config1_bit_exact(engine, idx):
    case = load_json("sieve.json")["cases"][idx]
    best = engine.run_sieve(case["r"], case["depth"], case["smax"])
    got = "".join(l + "\n" for l in engine.cert_lines(best))
    with gzip.open(os.path.join(GOLDEN, case["file"]), "rt") as f:
        assert got == f.read()


def test_sieve_gpu_selftest_config(engine, oracle):
    # coarse_sieve --selftest: r = 136279841, d <= 20, smax = 999999
    case = [c for c in load_json("sieve.json")["cases"] if c["smax"] == 999999][0]
    best = engine.run_sieve(136279841, 20, 999999)
    txt = "".join(l + "\n" for l in engine.cert_lines(best))
    assert sha(txt.encode()) == case["sha256"]
    assert (best == oracle.sieve(136279841, 20, 999999)).all()


def test_sieve_extend_from_preload(engine, oracle):
    r, smax = 44687, 22343
    lo = engine.run_sieve(r, 12, smax)
    full = engine.run_sieve(r, 20, smax, dmin=13, preload=lo)
    assert (full == oracle.sieve(r, 20, smax)).all()


def test_sieve_small_and_edge(engine, oracle):
    for r, depth, smax in [(101, 9, 100), (136279841, 11, 30000), (74207281, 10, 20000),
                           (7, 2, 3), (136279841, 24, 4000)]:
        assert (engine.run_sieve(r, depth, smax) == oracle.sieve(r, depth, smax)).all(), (r, depth)


def test_sieve_rejects_bad_r(engine):
    with pytest.raises(engine.Gf2eError) as e:
        engine.run_sieve(127, 7, 50)
    assert e.value.status == -4


def test_sieve_stats_match_oracle(engine, oracle):
    r, smax = 44687, 22343
    best = engine.DeviceBuffer(8 * (smax + 1))
    ws = engine.sieve_device(r, 20, smax, best)
    cls, mk = ws.stats()
    _, ocls, omk = oracle.sieve(r, 20, smax, stats=True)
    assert list(cls[2:21]) == list(ocls[2:21])
    assert list(mk[2:21]) == list(omk[2:21])


# ----------------------------------------------------------------- squaring
def _square_k(engine, st, r, s, k):
    a = engine.DeviceBuffer.from_array(st)
    b = engine.DeviceBuffer(a.nbytes)
    for _ in range(k):
        engine.trin_square(a, b, r, s)
        a, b = b, a
    return a.to_numpy(len(st))


def test_square_fixtures_single(engine, oracle):
    for c in load_json("square.json")["cases"]:
        if "words" not in c:          # hash-only cases: test_gpu_frobenius.py
            continue
        got = _square_k(engine, oracle.x_state(c["r"]), c["r"], c["s"], c["k"])
        assert (got == words_of(c["words"])).all(), c


def test_square_random_states_vs_oracle(engine, oracle):
    rng = np.random.default_rng(11)
    for r in (31, 127, 129, 4423, 999961, 136279841):
        for s in sorted({1, 2, 63, 64, 65, (r - 1) // 2, int(rng.integers(1, (r - 1) // 2 + 1))}):
            if not (1 <= s and 2 * s < r):
                continue
            st = rand_state(rng, r)
            k = 2 if r > 10**6 else 5
            want = oracle.trin_square_k(st, r, s, k)
            assert (_square_k(engine, st, r, s, k) == want).all(), (r, s)


def test_square_batch_mixed_s(engine, oracle):
    r = 4423
    ss = [1, 2, 63, 64, 65, 127, 128, 129, 1000, 2211, 1200, 7]
    nw = (r + 63) // 64
    stride = nw + (nw & 1)
    states = np.zeros(stride * len(ss), dtype=np.uint64)
    for i in range(len(ss)):
        states[i * stride] = 2
    dst = engine.DeviceBuffer.from_array(states)
    scr = engine.DeviceBuffer(dst.nbytes)
    ds = engine.DeviceBuffer.from_array(np.array(ss, dtype=np.uint64))
    engine.trin_square_batch(dst, scr, stride, len(ss), r, ds, 50)
    got = dst.to_numpy(stride * len(ss)).reshape(len(ss), stride)[:, :nw]
    cases = {(c["s"]): c for c in load_json("square.json")["cases"] if c["r"] == r and c["k"] == 50}
    for i, s in enumerate(ss):
        want = words_of(cases[s]["words"]) if s in cases else \
            oracle.trin_square_k(oracle.x_state(r), r, s, 50)
        assert (got[i] == want).all(), s


def test_square_config2_fixture_hashes(engine):
    fx = [c for c in load_json("square.json")["cases"] if c["k"] == 4096]
    r = fx[0]["r"]
    nw = (r + 63) // 64
    stride = nw + (nw & 1)
    n = len(fx)
    dst = engine.DeviceBuffer(8 * stride * n)
    scr = engine.DeviceBuffer(dst.nbytes)
    engine.trin_set_x(dst, stride, n, r)
    ds = engine.DeviceBuffer.from_array(np.array([c["s"] for c in fx], dtype=np.uint64))
    engine.trin_square_batch(dst, scr, stride, n, r, ds, 4096)
    got = dst.to_numpy(stride * n).reshape(n, stride)[:, :nw]
    for i, c in enumerate(fx):
        assert sha(np.ascontiguousarray(got[i]).tobytes()) == c["sha256"]


def test_reduce_vs_oracle(engine, oracle):
    rng = np.random.default_rng(2)
    for r, s in [(4423, 1200), (4423, 1), (4423, 2211), (127, 63), (999961, 400000)]:
        L = 2 * r - 1
        P = rand_state(rng, L)
        want = oracle.mod_trinomial(np.concatenate([P, np.zeros(2, np.uint64)]), L, r, s)
        dP = engine.DeviceBuffer.from_array(P)
        dO = engine.DeviceBuffer(8 * ((r + 63) // 64))
        engine.trin_reduce(dP, L, dO, r, s)
        assert (dO.to_numpy((r + 63) // 64) == want).all(), (r, s)


def test_square_rejects_bad_s(engine):
    a = engine.DeviceBuffer(8 * 70)
    b = engine.DeviceBuffer(8 * 70)
    for s in (0, 2212, 5000):
        with pytest.raises(engine.Gf2eError):
            engine.trin_square(a, b, 4423, s)


# ------------------------------------------------------------------- FFT
def test_fft_transform_fixtures(engine, oracle):
    for t in load_json("fft.json")["transforms"]:
        m = t["m"]
        f = W.splitmix64(t["seed"], 1 << m)
        F = engine.CudaFFT()
        F.init(m)
        d = engine.DeviceBuffer.from_array(f)
        F.fwd(d)
        g = d.to_numpy(1 << m)
        assert sha(g.tobytes()) == t["fwd_sha256"], m
        F.inv(d)
        assert (d.to_numpy(1 << m) == f).all(), m
        F.fini()


@pytest.mark.parametrize("m", [15, 16, 17, 18, 20])
def test_fft_transform_vs_oracle(engine, oracle, m):
    f = W.splitmix64(900 + m, 1 << m)
    F = engine.CudaFFT()
    F.init(m)
    d = engine.DeviceBuffer.from_array(f)
    F.fwd(d)
    assert (d.to_numpy(1 << m) == oracle.fft_fwd(f, m)).all()
    F.inv(d)
    assert (d.to_numpy(1 << m) == f).all()


@pytest.mark.parametrize("m", [22, 24])
def test_fft_large_roundtrip_and_linearity(engine, m):
    n = 1 << m
    f = W.splitmix64(31 + m, n)
    g = W.splitmix64(57 + m, n)
    F = engine.CudaFFT()
    F.init(m)
    df, dg, dh = (engine.DeviceBuffer.from_array(x) for x in (f, g, f ^ g))
    for d in (df, dg, dh):
        F.fwd(d)
    assert (df.to_numpy(n) ^ dg.to_numpy(n) == dh.to_numpy(n)).all()
    F.inv(df)
    assert (df.to_numpy(n) == f).all()


def test_twiddles_fixture(engine):
    F = engine.CudaFFT()
    F.init(10)
    assert sha(F.twiddles().tobytes()) == load_json("fft.json")["twiddles_m10_sha256"]


def test_product_fixtures(engine):
    for c in load_json("fft.json")["products"]:
        a = W.random_bits(c["abits"], c["seed_a"])
        b = W.random_bits(c["bbits"], c["seed_b"])
        out = engine.gf2x_fft_mul(a, c["abits"], b, c["bbits"])
        assert sha(out.tobytes()) == c["sha256"], (c["abits"], c["bbits"])


def test_mul_batch_uneven_vs_oracle(engine, oracle):
    sizes = [(1, 1), (5, 700), (4096, 33), (100000, 100000), (65537, 3), (2**18, 2**17 + 5)]
    bufs, jobs, wants = [], [], []
    for i, (ab, bb) in enumerate(sizes):
        a, b = W.random_bits(ab, 10 + i), W.random_bits(bb, 20 + i)
        da, db = engine.DeviceBuffer.from_array(a), engine.DeviceBuffer.from_array(b)
        do = engine.DeviceBuffer(8 * engine.mul_out_words(ab, bb))
        bufs += [da, db, do]
        jobs.append((da, ab, db, bb, do))
        wants.append(oracle.comb_mul(a, ab, b, bb))
    engine.mul_batch_dev(jobs)
    engine.stream_sync()
    for (da, ab, db, bb, do), want in zip(jobs, wants):
        assert (do.to_numpy(len(want)) == want).all(), (ab, bb)


def test_mul_batch_large_residues(engine, oracle):
    """Full-size operands (to 2^27 bits) checked by residues mod degree-61
    irreducibles, the reference's bigtest method (cantor_ref.cpp:159-224)."""
    cfg = W.mul_config(1, npairs=6, lo=24.0, hi=27.0)
    bufs, jobs = [], []
    for i, (ab, bb) in enumerate(cfg["sizes"]):
        a, b = W.random_bits(ab, 100 + i), W.random_bits(bb, 200 + i)
        da, db = engine.DeviceBuffer.from_array(a), engine.DeviceBuffer.from_array(b)
        do = engine.DeviceBuffer(8 * engine.mul_out_words(ab, bb))
        bufs.append((a, b))
        jobs.append((da, ab, db, bb, do))
    engine.mul_batch_dev(jobs)
    engine.stream_sync()
    q, d = _irreducible61(oracle)
    for (a, b), (da, ab, db, bb, do) in zip(bufs, jobs):
        out = do.to_numpy(engine.mul_out_words(ab, bb))
        lhs = oracle.modq_mul(oracle.residue(a, ab, q, d), oracle.residue(b, bb, q, d), q, d)
        assert lhs == oracle.residue(out, ab + bb, q, d), (ab, bb)


def _irreducible61(oracle):
    """Smallest irreducible x^61 + ... above a seed (ModP, gf2_cantor_engine.h:327-334).
    d = 61 is prime, so x^(2^61) == x mod q with q(0) = 1 suffices."""
    low = 0xC0FFEE | 1
    while True:
        q = (1 << 61) | (low & ((1 << 61) - 1))
        t = 2
        for _ in range(61):
            t = oracle.modq_mul(t, t, q, 61)
        if t == 2:
            return q, 61
        low += 2


# -------------------------------------------------------- TrinGPU context
def test_tringpu_interval_product_fixture(engine):
    p = load_json("square.json")["products"][0]
    G = engine.TrinGPU()
    G.init(p["r"])
    G.set_s(p["s"])
    G.set_x()
    G.reset_acc()
    for k in range(1, p["k1"] + 1):
        G.square_A()
        if k >= p["k0"]:
            G.accumulate()
    assert (G.read("ACC") == words_of(p["words"])).all()
    G.fini()


def test_tringpu_config2_product_fixture(engine):
    p = load_json("square.json")["products"][1]
    G = engine.TrinGPU()
    G.init(p["r"])
    G.set_s(p["s"])
    G.set_x()
    G.reset_acc()
    for k in range(1, p["k1"] + 1):
        G.square_A()
        if k >= p["k0"]:
            G.accumulate()
    assert sha(G.read("ACC").tobytes()) == p["sha256"]
    G.fini()


def test_spread_square_equals_fft_square(engine):
    """trinomial_stage2 bench cross-check: spread-square == FFT-square."""
    r, s = 999961, 12345
    G = engine.TrinGPU()
    G.init(r)
    G.set_s(s)
    G.set_x()
    for _ in range(30):
        G.square_A()
    G.mul_dev(G.dA, G.dA)
    G.reduce(G.dACC, 2 * r - 1)
    G.square_A()
    assert (G.read("A") == G.read("ACC")).all()
    G.fini()


# ------------------------------------------------ host-buffer squaring API
@pytest.mark.parametrize("r,n,k", [(999961, 8, 5), (136279841, 33, 3)])
def test_frobenius_host_vs_oracle(engine, oracle, r, n, k):
    """F_k = x^(2^k) for many s through host buffers; at r = 136279841 the
    33 states (561 MB) are squared in groups of 13, 16 and 4 states whose
    readbacks overlap the next group's squarings (states 0, 16 and 32 are
    checked: one from each group)."""
    rng = np.random.default_rng(r + n)
    s_values = rng.integers(3, r // 2, size=n).astype(np.uint64)
    got = engine.frobenius_host(r, s_values, k)
    for i in sorted({0, n // 2, n - 1, min(16, n - 1)}):
        want = oracle.trin_square_k(oracle.x_state(r), r, int(s_values[i]), k)
        assert (got[i][: want.size] == want).all(), i
