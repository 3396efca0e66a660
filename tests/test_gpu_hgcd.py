"""Subquadratic GPU gcd (half-gcd recursion) against the oracle's Euclid
(gf2_gcd.h:48-75) and the quadratic GPU gcd: planted common factors, edge
cases, scan accumulators against the trinomial, small thresholds that force
deep recursion and FFT products, lockstep batches (max_parallel >= 2: all
jobs stepped through the recursion together, members of very different
sizes and members that finish early) against one-at-a-time runs, and the
reference's known answer at r = 136279841 (s = 474: least factor
3991ef16129, degree 41)."""
import os

import numpy as np
import pytest

from mersenne_trinomial_b200 import workloads as W

pytestmark = pytest.mark.gpu


def exact_degree(v, d):
    v = v.copy()
    v[d >> 6] |= np.uint64(1 << (d & 63))
    return v


def trinomial(r, s):
    T = np.zeros((r + 1 + 63) // 64, dtype=np.uint64)
    for e in (0, s, r):
        T[e >> 6] |= np.uint64(1 << (e & 63))
    return T


@pytest.fixture
def thresholds():
    """Set the half-gcd thresholds for one test (read per gcd call)."""
    saved = {k: os.environ.get(k) for k in
             ("GF2E_HGCD_BASE_BITS", "GF2E_HGCD_SMALL_BITS", "GF2E_HGCD_FFT_BITS")}

    def set_(base=None, small=None, fft=None):
        for k, v in (("GF2E_HGCD_BASE_BITS", base), ("GF2E_HGCD_SMALL_BITS", small),
                     ("GF2E_HGCD_FFT_BITS", fft)):
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = str(v)
    yield set_
    for k, v in saved.items():
        if v is None:
            os.environ.pop(k, None)
        else:
            os.environ[k] = v


def run_pairs(engine, arrays, cap=0, par=1):
    keep, pairs = [], []
    for a, ab, b, bb in arrays:
        da, db = engine.DeviceBuffer.from_array(a), engine.DeviceBuffer.from_array(b)
        keep += [da, db]
        pairs.append((da, ab, db, bb))
    return engine.gcd_large(pairs, g_cap_words=cap, max_parallel=par)


def planted(oracle, rng, t, gd, ud, vd):
    g = exact_degree(W.random_bits(gd + 1, 100 + t), gd)
    u = exact_degree(W.random_bits(ud + 1, 200 + t), ud)
    v = exact_degree(W.random_bits(vd + 1, 300 + t), vd)
    a = oracle.comb_mul(g, gd + 1, u, ud + 1)
    b = oracle.comb_mul(g, gd + 1, v, vd + 1)
    return a, b


@pytest.mark.parametrize("par", [1, 5])
@pytest.mark.parametrize("base,small,fft", [(None, None, None), (256, 512, 2048),
                                            (512, 1024, 1 << 30), (4096, 8192, 4096)])
def test_hgcd_planted_factors(engine, oracle, thresholds, base, small, fft, par):
    thresholds(base, small, fft)
    rng = np.random.default_rng(11)
    arrays, want = [], []
    for t, (gd, ud, vd) in enumerate([(700, 30000, 29000), (5, 60000, 60000), (3000, 20000, 45000),
                                      (1, 100000, 99999), (40000, 30000, 1000)]):
        a, b = planted(oracle, rng, t, gd, ud, vd)
        arrays.append((a, 64 * a.size, b, 64 * b.size))
        want.append(oracle.poly_gcd(a, b))
    degs, gs, st = run_pairs(engine, arrays, cap=1200, par=par)
    for (wd, wg), d, g in zip(want, degs.tolist(), gs):
        assert d == wd
        n = min(len(wg), len(g))
        assert (g[:n] == wg[:n]).all() and not g[n:].any() and not wg[n:].any()
    if base is not None:
        assert st["nodes"] > st["base_cases"] > 0          # the recursion really ran


@pytest.mark.parametrize("par", [1, 8])
def test_hgcd_edge_cases(engine, oracle, thresholds, par):
    """Units, zeros, x, equal operands, swapped orders, b | a; in a lockstep
    batch these members finish at different steps."""
    thresholds(256, 512, 2048)
    one = np.array([1], dtype=np.uint64)
    zero = np.zeros(2, dtype=np.uint64)
    x = np.array([2], dtype=np.uint64)
    big = exact_degree(W.random_bits(50000, 9), 49999)
    big2 = exact_degree(W.random_bits(30000, 10), 29999)
    cases = [(one, 64, big, 50000), (zero, 128, big, 50000), (big, 50000, big, 50000),
             (x, 64, big, 50000), (big, 50000, zero, 128), (big2, 30000, big, 50000),
             (big, 50000, big2, 30000)]
    # b divides a
    prod = oracle.comb_mul(big2, 30000, big, 50000)
    cases.append((prod, 64 * prod.size, big2, 30000))
    arrays, want = [], []
    for a, ab, b, bb in cases:
        arrays.append((a, ab, b, bb))
        want.append(oracle.poly_gcd(a, b)[0])
    degs, _, _ = run_pairs(engine, arrays, par=par)
    assert degs.tolist() == want


@pytest.mark.parametrize("par", [1, 3])
def test_hgcd_matches_quadratic_gpu_gcd_on_trinomials(engine, thresholds, par):
    """gcd(ACC, T) at r ~ 2*10^5 for running products like the scan's, half-gcd
    vs the quadratic Lehmer gcd (both GPU; the latter is pinned to the oracle)."""
    thresholds(2048, 4096, 1 << 17)
    r = 200003
    arrays = []
    for s in (5, 1001, 77777):
        T = engine.TrinGPU()
        T.init(r)
        T.set_s(s)
        T.set_x()
        T.reset_acc()
        for k in range(1, 40):
            T.square_A()
            if k > 8:
                T.accumulate()
        acc = T.read("ACC")
        T.fini()
        arrays.append((acc, r, trinomial(r, s), r + 1))
    degs, gs, _ = run_pairs(engine, arrays, cap=64, par=par)
    keep, pairs = [], []
    for a, ab, b, bb in arrays:
        da, db = engine.DeviceBuffer.from_array(a), engine.DeviceBuffer.from_array(b)
        keep += [da, db]
        pairs.append((da, ab, db, bb))
    want, wgs = engine.gcd_batch(pairs, g_cap_words=64)
    assert degs.tolist() == want.tolist()
    for g, w in zip(gs, wgs):
        assert (g is None) == (w is None)
        if g is not None:
            assert (g == w).all()


def test_hgcd_concurrent_jobs_match_serial(engine, oracle):
    rng = np.random.default_rng(5)
    arrays = []
    for t in range(6):
        a, b = planted(oracle, rng, 40 + t, 100 + 50 * t, 70000 + 1000 * t, 69000)
        arrays.append((a, 64 * a.size, b, 64 * b.size))
    d1, g1, _ = run_pairs(engine, arrays, cap=64, par=1)
    d4, g4, _ = run_pairs(engine, arrays, cap=64, par=4)
    assert d1.tolist() == d4.tolist()
    for x, y in zip(g1, g4):
        assert (x == y).all()


def scan_accumulators(engine, r, ss, k1, k0):
    arrays = []
    for s in ss:
        T = engine.TrinGPU()
        T.init(r)
        T.set_s(s)
        T.set_x()
        T.reset_acc()
        for k in range(1, k1 + 1):
            T.square_A()
            if k >= k0:
                T.accumulate()
        arrays.append((T.read("ACC"), r, trinomial(r, s), r + 1))
        T.fini()
    return arrays


def test_lockstep_matches_single_at_default_thresholds(engine):
    """Sixteen interval gcds at r = 1000003 (default thresholds: base cases,
    schoolbook and FFT products, all batched) as two lockstep batches of
    eight running at once on two streams, as one batch of eight after
    another, and as batches of four, against one gcd at a time."""
    r = 1000003
    ss = [3, 12, 101, 4567, 33333, 77777, 250001, 499999,
          5, 77, 1234, 9999, 123457, 300007, 444443, 499001]
    arrays = scan_accumulators(engine, r, ss, 48, 20)
    d1, g1, _ = run_pairs(engine, arrays, cap=64, par=1)
    for par in (16, 8, 4):
        dp, gp, st = run_pairs(engine, arrays, cap=64, par=par)
        assert dp.tolist() == d1.tolist(), par
        for x, y in zip(g1, gp):
            assert (x is None) == (y is None)
            if x is not None:
                assert (x == y).all()
        assert st["base_cases"] > 0 and st["fft_products"] > 0


@pytest.mark.timeout(900)
def test_hgcd_kat_r136279841_s474(engine, oracle):
    """The reference's known answer `474 41 p3991ef16129` at r = 136279841
    (tsfactor_handoff.md:337): ACC = prod_{k=25}^{88} (x^(2^k) + x) mod T,
    g = gcd(ACC, T) on the GPU; its least factor is the certificate's."""
    r, s = 136279841, 474
    T = engine.TrinGPU()
    T.init(r)
    T.set_s(s)
    T.set_x()
    T.reset_acc()
    for k in range(1, 89):
        T.square_A()
        if k >= 25:
            T.accumulate()
    acc = T.read("ACC")
    T.fini()
    degs, gs, st = run_pairs(engine, [(acc, r, trinomial(r, s), r + 1)], cap=64, par=1)
    g = gs[0]
    assert degs[0] >= 41 and g is not None
    d, mask = engine.resolve_factor(g, 25, 88)
    assert d == 41 and engine.engine._hex(mask) == "3991ef16129"
    assert oracle.factor_divides(r, s, 41, "3991ef16129") == 1
