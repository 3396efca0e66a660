"""Host-side hit resolution (gf2e_resolve_factor): least factor degree and
the numerically least factor of that degree, on gcds built from known
irreducible factors and on gcds taken from the oracle's deep scan
(trinomial_scan.cu:283-325, gf2_gcd_ntl.cpp:68-92).  CPU only."""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, ROOT)


def _words(v: int) -> np.ndarray:
    n = max(1, (v.bit_length() + 63) // 64)
    return np.array([(v >> (64 * i)) & 0xFFFFFFFFFFFFFFFF for i in range(n)], dtype=np.uint64)


def _int(w) -> int:
    return sum(int(x) << (64 * i) for i, x in enumerate(np.asarray(w, dtype=np.uint64).tolist()))


def _mul(a: int, b: int) -> int:
    out = 0
    while b:
        if b & 1:
            out ^= a
        a <<= 1
        b >>= 1
    return out


def _mod(a: int, m: int) -> int:
    dm = m.bit_length()
    while a.bit_length() >= dm:
        a ^= m << (a.bit_length() - dm)
    return a


def _irreducible(p: int) -> bool:
    """Rabin's test: x^(2^d) = x mod p and gcd(x^(2^(d/q)) - x, p) = 1."""
    d = p.bit_length() - 1
    if d < 1:
        return False

    def x2k(k):
        h = 2
        for _ in range(k):
            h = _mod(_mul(h, h), p)
        return h

    def gcd(a, b):
        while b:
            a, b = b, _mod(a, b)
        return a

    if x2k(d) != _mod(2, p):
        return False
    q, n, primes = 2, d, []
    while q * q <= n:
        if n % q == 0:
            primes.append(q)
            while n % q == 0:
                n //= q
        q += 1
    if n > 1:
        primes.append(n)
    return all(gcd(x2k(d // q) ^ 2, p) == 1 for q in primes)


def _irreducibles(d: int, count: int, start: int = 0):
    out = []
    for low in range(start, 1 << d):
        p = (1 << d) | low
        if low & 1 and _irreducible(p):
            out.append(p)
            if len(out) == count:
                break
    return out


def _tri(r: int, s: int) -> int:
    return (1 << r) | (1 << s) | 1


@pytest.fixture(scope="module")
def M():
    import mersenne_trinomial_b200 as M
    return M


def _resolve(M, g: int, kmax: int):
    d, mask = M.resolve_factor(_words(g), 1, kmax, cap=_words(g).size + 2)
    return d, _int(mask)


def test_least_degree_of_mixed_product(M):
    f5, f7, f13 = _irreducibles(5, 1)[0], _irreducibles(7, 1)[0], _irreducibles(13, 1)[0]
    g = _mul(_mul(f7, f13), f5)
    assert _resolve(M, g, 64) == (5, f5)


def test_equal_degree_split_takes_the_least(M):
    fs = _irreducibles(9, 3, start=37)
    g = _mul(_mul(fs[2], fs[0]), fs[1])
    assert _resolve(M, g, 64) == (9, min(fs))


@pytest.mark.parametrize("r,s", [(607, 273), (1279, 418), (2281, 715)])
def test_irreducible_trinomial_is_its_own_factor(M, r, s):
    g = _tri(r, s)
    assert _resolve(M, g, r + 10) == (r, g)


def test_large_factor_behind_small_one(M):
    # x^521 + x^32 + 1 and x^607 + x^273 + 1 are irreducible; a degree-11
    # factor in the product is found first
    f11 = _irreducibles(11, 1, start=200)[0]
    g = _mul(_mul(_tri(607, 273), _tri(521, 32)), f11)
    assert _resolve(M, g, 700) == (11, f11)
    g2 = _mul(_tri(607, 273), _tri(521, 32))
    assert _resolve(M, g2, 700) == (521, _tri(521, 32))


def test_no_factor_up_to_kmax_is_an_error(M):
    from mersenne_trinomial_b200 import Gf2eError
    with pytest.raises(Gf2eError):
        _resolve(M, _tri(607, 273), 600)


def test_matches_oracle_scan_gcds(M, oracle):
    r, seen = 4423, 0
    for s in range(3, 400):
        st, d, gdeg, g_hex, mask_hex = oracle.scan_one(r, s, 1, 40)
        if st != 1 or mask_hex is None:
            continue
        g = int(g_hex, 16)
        assert _resolve(M, g, 40) == (d, int(mask_hex, 16)), s
        seen += 1
        if seen == 12:
            break
    assert seen == 12


def test_portable_clmul_path_agrees():
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "import numpy as np, mersenne_trinomial_b200 as M\n"
        "g = (1 << 1279) | (1 << 418) | 1\n"
        "w = np.array([(g >> (64 * i)) & ((1 << 64) - 1) for i in range(20)], dtype=np.uint64)\n"
        "d, m = M.resolve_factor(w, 1, 1300, cap=24)\n"
        "print(d, sum(int(x) << (64 * i) for i, x in enumerate(m.tolist())) == g)\n" % ROOT)
    env = dict(os.environ, GF2E_NO_PCLMUL="1")
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr
    assert out.stdout.split() == ["1279", "True"]
