"""Batched repeated squaring with two squarings per pass (F -> F^4 mod T in
one read and one write of every state) against the oracle and the
reference's own kernels, through the C ABI.  Bit-exact: GF(2) arithmetic.

gf2e_trin_square_batch runs floor(k/2) fused passes (plus single passes for
an odd k, or to make the pass count even), so k = 2..7 cover every pass mix;
the one-squaring kernel is checked separately by the single-state entry
point (gf2e_trin_square, one squaring per call)."""
import hashlib

import numpy as np
import pytest

from conftest import load_json

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def fused_everywhere(monkeypatch):
    """Small batches would take the one-squaring pass (they fit in L2): force
    the fused pass so that every case here exercises it."""
    monkeypatch.setenv("GF2E_SQUARINGS_PER_PASS", "2")


def rand_states(rng, r, n):
    nw = (r + 63) // 64
    st = rng.integers(0, 2**63, size=(n, nw), dtype=np.uint64) * np.uint64(2) + \
        rng.integers(0, 2, size=(n, nw), dtype=np.uint64)
    if r & 63:
        st[:, -1] &= np.uint64((1 << (r & 63)) - 1)
    return st


def square_batch(engine, states, r, ss, k):
    n, nw = states.shape
    stride = nw + (nw & 1)
    buf = np.zeros((n, stride), dtype=np.uint64)
    buf[:, :nw] = states
    dst = engine.DeviceBuffer.from_array(buf.reshape(-1))
    scr = engine.DeviceBuffer(dst.nbytes)
    ds = engine.DeviceBuffer.from_array(np.asarray(ss, dtype=np.uint64))
    engine.trin_square_batch(dst, scr, stride, n, r, ds, k)
    return dst.to_numpy(n * stride).reshape(n, stride)[:, :nw]


def square_single_passes(engine, st, r, s, k):
    a = engine.DeviceBuffer.from_array(st)
    b = engine.DeviceBuffer(a.nbytes)
    for _ in range(k):
        engine.trin_square(a, b, r, s)
        a, b = b, a
    return a.to_numpy(len(st))


@pytest.mark.parametrize("r", [5, 7, 31, 127, 129, 191, 193, 255, 257, 4423])
def test_every_s_random_states(engine, oracle, r):
    """Every admissible s of small r (all window layouts, word-boundary and
    one-word states), k = 2..7, from random states."""
    rng = np.random.default_rng(r)
    ss = list(range(1, (r - 1) // 2 + 1))
    for k in (2, 3, 4, 5, 6, 7):
        st = rand_states(rng, r, len(ss))
        got = square_batch(engine, st, r, ss, k)
        for i, s in enumerate(ss):
            assert (got[i] == oracle.trin_square_k(st[i], r, s, k)).all(), (r, s, k)


def test_word_boundary_s_mid_r(engine, oracle):
    rng = np.random.default_rng(7)
    for r in (8191 * 8 + 1 + 2, 65537, 999961):
        h = (r - 1) // 2
        ss = sorted({1, 2, 3, 31, 32, 33, 63, 64, 65, 127, 128, 129, 1000, h // 3, h // 2,
                     h - 64, h - 1, h, int(rng.integers(1, h + 1))})
        st = rand_states(rng, r, len(ss))
        for k in (2, 3, 8):
            got = square_batch(engine, st, r, ss, k)
            for i, s in enumerate(ss):
                assert (got[i] == oracle.trin_square_k(st[i], r, s, k)).all(), (r, s, k)


def test_full_size_r_against_oracle_and_single_passes(engine, oracle):
    """r = 136279841 (17 MB states): s = 1, 63, 64, 65, (r-1)/2 and the
    reference's certificate s = 474, from random states."""
    r = 136279841
    rng = np.random.default_rng(136)
    ss = [1, 63, 64, 65, 474, 7458, 2000000, (r - 1) // 3, (r - 1) // 2]
    st = rand_states(rng, r, len(ss))
    got2 = square_batch(engine, st, r, ss, 2)
    got3 = square_batch(engine, st[:3], r, ss[:3], 3)
    for i, s in enumerate(ss):
        want = oracle.trin_square_k(st[i], r, s, 2)
        assert (got2[i] == want).all(), s
        if i < 2:
            assert (square_single_passes(engine, st[i], r, s, 2) == want).all(), s
        if i < 3:
            assert (got3[i] == oracle.trin_square_k(st[i], r, s, 3)).all(), s


def test_reference_fixtures_full_size_r(engine):
    """x^(2^k) mod T at r = 136279841 as the reference's own squaring kernels
    compute it (run under their CPU emulation): k = 3 at word-boundary s,
    and k = 256 for the benchmark's first two s values."""
    cases = [c for c in load_json("square.json")["cases"] if c["r"] == 136279841]
    assert len(cases) >= 8
    r = 136279841
    nw = (r + 63) // 64
    stride = nw + (nw & 1)
    for k in sorted({c["k"] for c in cases}):
        cs = [c for c in cases if c["k"] == k]
        n = len(cs)
        dst = engine.DeviceBuffer(8 * stride * n)
        scr = engine.DeviceBuffer(dst.nbytes)
        engine.trin_set_x(dst, stride, n, r)
        ds = engine.DeviceBuffer.from_array(np.array([c["s"] for c in cs], dtype=np.uint64))
        engine.trin_square_batch(dst, scr, stride, n, r, ds, k)
        got = dst.to_numpy(stride * n).reshape(n, stride)[:, :nw]
        for i, c in enumerate(cs):
            h = hashlib.sha256(np.ascontiguousarray(got[i]).tobytes()).hexdigest()
            assert h == c["sha256"], (c["s"], k)
