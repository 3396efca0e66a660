"""GPU gcd (one thread block per pair) against the oracle's naive Euclid
(gf2_gcd.h:48-75), with planted common factors and the scan's real operands
(interval accumulators against the trinomial)."""
import numpy as np
import pytest

from mersenne_trinomial_b200 import workloads as W

pytestmark = pytest.mark.gpu


def trinomial(r, s):
    T = np.zeros((r + 1 + 63) // 64, dtype=np.uint64)
    for e in (0, s, r):
        T[e >> 6] |= np.uint64(1 << (e & 63))
    return T


def exact_degree(v, d):
    v = v.copy()
    v[d >> 6] |= np.uint64(1 << (d & 63))
    return v


def test_gcd_planted_factors(engine, oracle):
    rng = np.random.default_rng(4)
    pairs, keep, want = [], [], []
    for t in range(24):
        gd = int(rng.integers(1, 3000))
        ud, vd = int(rng.integers(1, 9000)), int(rng.integers(1, 9000))
        g = exact_degree(W.random_bits(gd + 1, 100 + t), gd)
        u = exact_degree(W.random_bits(ud + 1, 200 + t), ud)
        v = exact_degree(W.random_bits(vd + 1, 300 + t), vd)
        a = oracle.comb_mul(g, gd + 1, u, ud + 1)
        b = oracle.comb_mul(g, gd + 1, v, vd + 1)
        wd, wg = oracle.poly_gcd(a, b)
        da, db = engine.DeviceBuffer.from_array(a), engine.DeviceBuffer.from_array(b)
        keep += [da, db]
        pairs.append((da, 64 * a.size, db, 64 * b.size))
        want.append((wd, wg))
    degs, gs = engine.gcd_batch(pairs, g_cap_words=200)
    for (wd, wg), d, g in zip(want, degs.tolist(), gs):
        assert d == wd
        n = min(len(wg), len(g))
        assert (g[:n] == wg[:n]).all() and not g[n:].any() and not wg[n:].any()


def test_gcd_edge_cases(engine, oracle):
    one = np.array([1], dtype=np.uint64)
    zero = np.zeros(2, dtype=np.uint64)
    x = np.array([2], dtype=np.uint64)
    big = W.random_bits(5000, 9)
    cases = [(one, 64, big, 5000), (zero, 128, big, 5000), (big, 5000, big, 5000),
             (x, 64, big, 5000), (zero, 128, zero, 128), (big, 5000, zero, 128)]
    keep, pairs, want = [], [], []
    for a, ab, b, bb in cases:
        da, db = engine.DeviceBuffer.from_array(a), engine.DeviceBuffer.from_array(b)
        keep += [da, db]
        pairs.append((da, ab, db, bb))
        want.append(oracle.poly_gcd(a, b)[0])
    degs, _ = engine.gcd_batch(pairs)
    assert degs.tolist() == want


def test_gcd_of_scan_accumulators(engine, oracle):
    """gcd(ACC, T) for interval products at r = 4423 (trinomial_scan's check)."""
    r = 4423
    keep, pairs, want = [], [], []
    for s in (3, 10, 13, 19, 1200, 2211):
        F = oracle.x_state(r)
        acc = np.zeros(oracle.words(r), dtype=np.uint64)
        acc[0] = 1
        for k in range(1, 61):
            F = oracle.trin_square_k(F, r, s, 1)
            if k > 5:
                t = F.copy()
                t[0] ^= np.uint64(2)
                acc = oracle.mod_trinomial(oracle.comb_mul(acc, r, t, r), 2 * r - 1, r, s)
        T = trinomial(r, s)
        want.append(oracle.poly_gcd(acc, T))
        da, db = engine.DeviceBuffer.from_array(acc), engine.DeviceBuffer.from_array(T)
        keep += [da, db]
        pairs.append((da, r, db, r + 1))
    degs, gs = engine.gcd_batch(pairs, g_cap_words=80)
    for (wd, wg), d, g in zip(want, degs.tolist(), gs):
        assert d == wd
        if d > 0:
            assert (g[:len(wg)] == wg[:len(g)]).all()


@pytest.mark.parametrize("r", [99991, 999961])
def test_gcd_large_random(engine, oracle, r):
    rng = np.random.default_rng(r)
    a = W.random_bits(r, 1)
    g = exact_degree(W.random_bits(40, 2), 39)
    b = oracle.comb_mul(W.random_bits(r - 50, 3), r - 50, g, 40)
    a = oracle.comb_mul(W.random_bits(r - 60, 4), r - 60, g, 40)
    wd, wg = oracle.poly_gcd(a, b)
    da, db = engine.DeviceBuffer.from_array(a), engine.DeviceBuffer.from_array(b)
    degs, gs = engine.gcd_batch([(da, 64 * a.size, db, 64 * b.size)], g_cap_words=4)
    assert degs[0] == wd and wd >= 39
    if wd < 256:
        assert (gs[0] == wg[:4]).all()
