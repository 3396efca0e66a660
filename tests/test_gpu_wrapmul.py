"""Products one transform size smaller with the wrapped part put back
(csrc/wrapmul.cu): the 2^m transform returns A B mod Z(y), Z the subspace
polynomial, and the top part floor(a b / x^T) from a small product restores
the rest.  Checked against the oracle's products for sizes just above a
power of two (equal, uneven, a square), through the TrinGPU context's
running product at an r whose r-bit products wrap, and through the batch
API with ordinary sizes mixed in."""
import numpy as np
import pytest

from mersenne_trinomial_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _dev(engine, words):
    return engine.DeviceBuffer.from_array(np.ascontiguousarray(words, dtype=np.uint64))


# (abits, bbits): chunk counts 2^16 + a little (m = 16 instead of 17), an
# uneven pair, wrapped parts of 1/10, 1/5 and 2/7 of 2^16 (the last beyond
# the 1/4 limit, so a plain product), and an ordinary size
SIZES = [(1 << 20 | 5000, 1 << 20 | 3000), ((1 << 21) - 64, 4000), (1 << 20 | 200000, 1 << 20),
         ((1 << 20) + 400000, 1 << 20), ((1 << 20) + 600000, 1 << 20), (300_000, 200_000)]


def test_batch_products_vs_oracle(engine, oracle):
    bufs, jobs, want = [], [], []
    for i, (ab, bb) in enumerate(SIZES):
        a = W.random_bits(ab, 40 + i)
        b = W.random_bits(bb, 80 + i)
        da, db = _dev(engine, a), _dev(engine, b)
        out = engine.DeviceBuffer(8 * engine.mul_out_words(ab, bb))
        bufs += [da, db, out]
        jobs.append((da, ab, db, bb, out))
        want.append(oracle.fft_mul(a, ab, b, bb))
    ws = engine.mul_batch_dev(jobs)
    for (da, ab, db, bb, out), w in zip(jobs, want):
        got = out.to_numpy(engine.mul_out_words(ab, bb))
        assert (got[: w.size] == w).all(), (ab, bb)
    # a second call on the same workspace gives the same products
    engine.mul_batch_dev(jobs, workspace=ws)
    for (da, ab, db, bb, out), w in zip(jobs, want):
        assert (out.to_numpy(engine.mul_out_words(ab, bb))[: w.size] == w).all()


def test_wrapped_square_vs_oracle(engine, oracle):
    ab = (1 << 20) + 777
    a = W.random_bits(ab, 5)
    da = _dev(engine, a)
    out = engine.DeviceBuffer(8 * engine.mul_out_words(ab, ab))
    engine.mul_batch_dev([(da, ab, da, ab, out)])
    w = oracle.fft_mul(a, ab, a, ab)
    assert (out.to_numpy(engine.mul_out_words(ab, ab))[: w.size] == w).all()


def test_tringpu_running_product_wraps(engine, oracle):
    # r-bit products with 2 * 8255 - 1 = 16509 chunks: a 2^14 transform
    r, s, k1 = 264149, 12345, 6
    G = engine.TrinGPU()
    G.init(r)
    G.set_s(s)
    G.set_x()
    G.reset_acc()
    F = oracle.x_state(r)
    acc = np.zeros_like(F)
    acc[0] = 1
    for k in range(1, k1 + 1):
        G.square_A()
        G.accumulate()
        F = oracle.trin_square_k(F, r, s, 1)
        Fx = F.copy()
        Fx[0] ^= np.uint64(2)
        prod = oracle.fft_mul(acc, r, Fx, r)
        acc = oracle.mod_trinomial(prod, 2 * r - 1, r, s)
    assert (G.read("ACC") == acc).all()
    G.fini()
