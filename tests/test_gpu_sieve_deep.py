"""The sieve at degrees 32..40 on the wide path (64-bit field elements, the
log table in value slices sized to the workspace; the reference's
coarse_sieve_wide, coarse_sieve.cu:920-1117 with gf2_wide_field.h).

Pinned two ways: the wide kernels run on degrees the dense path also covers
(GF2E_SIEVE_WIDE_FROM) and must give the same best[] and statistics, with
one slice and with many; and at r = 136279841 over every s <= (r-1)/2 the
survivor counts after each degree 32..36 are the reference's published ones
(coarse_sieve.log: 3731849, 3620029, 3515197, 3415883, 3322198), with a
sample of the new factors re-verified (check-ntl restatement) and tested
irreducible."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

R = 136279841
NONE = np.uint64(0xFFFFFFFFFFFFFFFF)


class _env:
    def __init__(self, **kw):
        self.kw = kw

    def __enter__(self):
        self.old = {k: os.environ.get(k) for k in self.kw}
        os.environ.update({k: str(v) for k, v in self.kw.items()})

    def __exit__(self, *a):
        for k, v in self.old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def _sieve(engine, r, dmin, dmax, smax, preload=None):
    best = engine.DeviceBuffer(8 * (smax + 1))
    if preload is not None:
        best.upload(preload)
    ws = engine.sieve_device(r, dmax, smax, best, dmin=dmin, fill=preload is None)
    out = best.to_numpy(smax + 1)
    cls, mk = ws.stats()
    return out, cls, mk


def _irreducible(p: int) -> bool:
    def mulmod(a, b):
        r = 0
        while b:
            if b & 1:
                r ^= a
            a <<= 1
            b >>= 1
            if a >> d & 1:
                a ^= p
        return r

    d = p.bit_length() - 1

    def x2k(k):
        h = 2
        for _ in range(k):
            h = mulmod(h, h)
        return h

    def gcd(a, b):
        while b:
            while a and a.bit_length() >= b.bit_length():
                a ^= b << (a.bit_length() - b.bit_length())
            a, b = b, a
        return a

    if x2k(d) != 2:
        return False
    n, q, primes = d, 2, []
    while q * q <= n:
        if n % q == 0:
            primes.append(q)
            while n % q == 0:
                n //= q
        q += 1
    if n > 1:
        primes.append(n)
    return all(gcd(x2k(d // q) ^ 2, p) == 1 for q in primes)


@pytest.mark.parametrize("budget_gb", [64, 0.25])
def test_wide_path_equals_dense_path(engine, budget_gb):
    """Degrees 16..31 through the wide kernels (one log-table slice, then
    0.25 GB slices: 32 of them at d = 31) against the dense tables."""
    smax = 2_000_000
    dense, c0, m0 = _sieve(engine, R, 2, 31, smax)
    with _env(GF2E_SIEVE_WIDE_FROM=16, GF2E_SIEVE_WIDE_GB=budget_gb):
        wide, c1, m1 = _sieve(engine, R, 2, 31, smax)
    assert (dense == wide).all()
    assert (c0 == c1).all() and (m0 == m1).all()


def test_wide_degrees_reject_out_of_range(engine):
    with pytest.raises(engine.Gf2eError):
        engine.engine.SieveWorkspace(41)


@pytest.mark.timeout(900)
def test_published_counts_d32_to_d36(engine, oracle):
    smax = (R - 1) // 2
    best, _, _ = _sieve(engine, R, 2, 31, smax)
    assert int(np.count_nonzero(best[1:] == NONE)) == 3849633
    want = {32: 3731849, 33: 3620029, 34: 3515197, 35: 3415883, 36: 3322198}
    rng = np.random.default_rng(36)
    for d in range(32, 37):
        before = best[1:] == NONE
        best, cls, mk = _sieve(engine, R, d, d, smax, preload=best)
        body = best[1:]
        assert int(np.count_nonzero(body == NONE)) == want[d], d
        new = np.nonzero(before & (body != NONE))[0]
        assert ((body[new] >> np.uint64(48)) == d).all()
        for i in rng.choice(new, size=min(8, new.size), replace=False):
            s = int(i) + 1
            mask = int(body[i]) & 0xFFFFFFFFFFFF
            assert oracle.factor_divides(R, s, d, format(mask, "x")) == 1, (s, d)
            assert _irreducible(mask), (s, d, hex(mask))
