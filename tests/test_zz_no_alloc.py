"""gf2e_mul_noalloc: the product entry point that allocates nothing per call,
for callers that cannot allocate device memory while they run (an HBM budget
reserved at start-up, or a loop that must not let an allocator synchronise
the device).  Its scratch is a fixed array inside the library, shared by all
calls, so this test checks it against the allocating gf2e_mul on two calls in
a row, through the C ABI.  The file name makes pytest collect it last."""
import ctypes

import numpy as np
import pytest

from mersenne_trinomial_b200 import workloads as W

pytestmark = pytest.mark.gpu

SIZES = [(1, 1), (100, 77), (4096, 4096), (100000, 77777), (2**22, 2**22 - 5)]


def _product_ref(M, a, ab, b, bb):
    """The existing entry point: gf2e_mul with its own plan and scratch."""
    F = M.CudaFFT()
    F.init(M.engine.fft_m_for(ab, bb))
    da, db = M.DeviceBuffer.from_array(a), M.DeviceBuffer.from_array(b)
    out = M.DeviceBuffer(8 * M.mul_out_words(ab, bb))
    fa, fb = M.DeviceBuffer(8 << F.m), M.DeviceBuffer(8 << F.m)
    M.gf2x_fft_mul_dev(F, da, ab, db, bb, out, fa, fb)
    res = out.to_numpy(M.mul_out_words(ab, bb))
    F.fini()
    return res


def _product_noalloc(M, da, ab, db, bb, out):
    st = M.lib().gf2e_mul_noalloc(da.ptr, ab, db.ptr, bb, out.ptr, None)
    M._lib.check(st)
    return out.to_numpy(M.mul_out_words(ab, bb))


def test_noalloc_matches_allocating_entry_two_calls(engine):
    M = engine
    for i, (ab, bb) in enumerate(SIZES):
        a1, b1 = W.random_bits(ab, 31 + i), W.random_bits(bb, 57 + i)
        a2, b2 = W.random_bits(ab, 91 + i), W.random_bits(bb, 13 + i)
        want1 = _product_ref(M, a1, ab, b1, bb)
        want2 = _product_ref(M, a2, ab, b2, bb)
        da1, db1 = M.DeviceBuffer.from_array(a1), M.DeviceBuffer.from_array(b1)
        da2, db2 = M.DeviceBuffer.from_array(a2), M.DeviceBuffer.from_array(b2)
        out = M.DeviceBuffer(8 * M.mul_out_words(ab, bb))
        # two calls in a row on the shared scratch, different operands, then
        # the first operands again: each must equal the allocating entry point
        got1 = _product_noalloc(M, da1, ab, db1, bb, out)
        got2 = _product_noalloc(M, da2, ab, db2, bb, out)
        got1b = _product_noalloc(M, da1, ab, db1, bb, out)
        assert (got1 == want1).all(), (ab, bb)
        assert (got2 == want2).all(), (ab, bb)
        assert (got1b == want1).all(), (ab, bb)
        if ab * bb <= 10**10:
            # and against the oracle's schoolbook product where that is quick
            from oracle import oracle as O
            assert (got2 == O.comb_mul(a2, ab, b2, bb)).all(), (ab, bb)


def test_noalloc_rejects_products_beyond_the_fixed_scratch(engine):
    M = engine
    L = M.lib()
    ab = bb = 2**22 + 64          # needs a transform of 2^19 points
    da = M.DeviceBuffer(8 * ((ab + 63) // 64))
    db = M.DeviceBuffer(8 * ((bb + 63) // 64))
    out = M.DeviceBuffer(8 * M.mul_out_words(ab, bb))
    assert L.gf2e_mul_noalloc(da.ptr, ab, db.ptr, bb, out.ptr, None) == -1
    assert b"2^18" in L.gf2e_last_error()
    assert L.gf2e_mul_noalloc(da.ptr, 0, db.ptr, bb, out.ptr, None) == -1
