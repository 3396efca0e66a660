"""The C-ABI library loads on a machine without a GPU, exports every symbol
include/*.h declares, and rejects bad arguments before touching the device
(the reference exit(1)s in those places; the library returns a status)."""
import glob
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names.update(re.findall(r"\b(gf2e_\w+)\s*\(", src))
    return sorted(names)


def test_header_symbols_exported(engine):
    import ctypes
    L = ctypes.CDLL(engine._lib.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) > 30
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_binding_covers_header(engine):
    from mersenne_trinomial_b200._lib import SIGNATURES
    assert set(declared_symbols()) <= set(SIGNATURES), set(declared_symbols()) - set(SIGNATURES)


def test_abi_version_and_status_strings(engine):
    L = engine.lib()
    assert L.gf2e_abi_version() == 1
    for st in range(0, -8, -1):
        assert L.gf2e_status_string(st)


def test_host_side_helpers_match_oracle(engine, oracle):
    for d in range(2, 25):
        assert engine.primitive_poly(d) == oracle.lib().orc_find_primitive_poly(d)
    B = engine.CantorBasis()
    B.build()
    assert B.len == 64 and B.verify()
    assert (B.b == oracle.cantor_basis()).all()
    for ab, bb in [(1, 1), (33, 31), (4096, 4096), (2**27, 2**27), (100, 2**20)]:
        assert engine.engine.fft_m_for(ab, bb) == oracle.lib().orc_fft_m_for(ab, bb)
        assert engine.mul_out_words(ab, bb) == oracle.mul_out_words(ab, bb)


def test_argument_errors_without_device(engine):
    L = engine.lib()
    # bad s for the trinomial (gf2_trinomial_cuda.h:118-123)
    assert L.gf2e_trin_square(8, 16, 4423, 0, None) == -1
    assert L.gf2e_trin_square(8, 16, 4423, 2212, None) == -1
    assert L.gf2e_trin_square(8, 16, 4424, 5, None) == -1          # even r
    assert b"s <=" in L.gf2e_last_error() or b"r must" in L.gf2e_last_error()
    # sieve degree range and workspace size
    assert L.gf2e_sieve_run(44687, 2, 41, 100, 8, 8, 1 << 30, None) == -1   # d <= 40
    assert L.gf2e_sieve_run(44687, 2, 20, 100, 8, 8, 16, None) == -1
    # FFT plan range
    import ctypes
    p = ctypes.c_void_p()
    assert L.gf2e_fft_plan_create(0, ctypes.byref(p)) == -1
    assert L.gf2e_fft_plan_create(31, ctypes.byref(p)) == -1


def test_unsupported_r_detected_on_host(engine):
    """gcd(r, 2^d-1) != 1 is refused before any launch (sieve_ref.cpp:79-83)."""
    L = engine.lib()
    assert L.gf2e_sieve_run(127, 2, 7, 50, 8, 8, 1 << 40, None) == -4
    assert b"gcd" in L.gf2e_last_error()


def test_workloads_are_seeded_and_valid():
    from mersenne_trinomial_b200 import workloads as W
    c1 = W.sieve_config(1)
    assert 40000 <= c1["r"] <= 50000 and c1["r"] % 8 in (1, 7) and W.is_prime(c1["r"])
    assert c1 == W.sieve_config(1)
    c2 = W.squaring_config(1)
    assert c2["r"] % 8 in (1, 7) and W.is_prime(c2["r"]) and len(c2["s"]) == 256
    assert (c2["s"] >= 3).all() and (c2["s"] <= c2["r"] // 2).all()
    c3 = W.mul_config(1)
    assert len(c3["sizes"]) == 64
    assert all(2**16 <= a <= 2**27 and 2**16 <= b <= 2**27 for a, b in c3["sizes"])
    x = W.random_bits(1000, 5)
    assert x.size == 16 and int(x[-1]) >> 40 == 0


def test_squarings_per_pass_rule(monkeypatch):
    """Host-only: the fused two-squaring pass is chosen for batches that do
    not fit in L2 (states and scratch above 96 MB), the one-squaring pass for
    smaller ones, r near 2^31 or an odd stride; GF2E_SQUARINGS_PER_PASS
    forces either."""
    import mersenne_trinomial_b200 as M
    L = M.lib()
    monkeypatch.delenv("GF2E_SQUARINGS_PER_PASS", raising=False)
    r = 136279841
    nw = (r + 63) // 64
    stride = nw + (nw & 1)
    assert L.gf2e_trin_squarings_per_pass(r, stride, 64) == 2
    assert L.gf2e_trin_squarings_per_pass(r, stride, 2) == 1          # 68 MB: in L2
    assert L.gf2e_trin_squarings_per_pass(r, stride + 1, 64) == 1     # odd stride
    assert L.gf2e_trin_squarings_per_pass(999961, 15626, 256) == 1    # config 2: 64 MB
    assert L.gf2e_trin_squarings_per_pass((1 << 31) - 1, 1 << 25, 8) == 1
    monkeypatch.setenv("GF2E_SQUARINGS_PER_PASS", "2")
    assert L.gf2e_trin_squarings_per_pass(999961, 15626, 256) == 2
    assert L.gf2e_trin_squarings_per_pass(r, stride + 1, 64) == 1
    monkeypatch.setenv("GF2E_SQUARINGS_PER_PASS", "1")
    assert L.gf2e_trin_squarings_per_pass(r, stride, 64) == 1
