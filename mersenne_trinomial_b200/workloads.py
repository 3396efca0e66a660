"""Seeded synthetic workloads with the shapes of the benchmark configurations.

  sieve_config(seed)       r: a prime = +-1 (mod 8) in [40000, 50000]; s = 1..r//2
                           except 2; degrees 2..20
  squaring_config(seed)    r: a prime = +-1 (mod 8) near 1,000,000; 256 s values
                           uniform in [3, r//2]; 4096 squarings from x
  mul_config(seed)         64 products, operand bit lengths floor(2^U),
                           U ~ Uniform[16, 27], uniform random bits (SplitMix64)
"""
from __future__ import annotations

import numpy as np

R_DEEP = 136279841


def is_prime(n: int) -> bool:
    if n < 2:
        return False
    if n % 2 == 0:
        return n == 2
    f = 3
    while f * f <= n:
        if n % f == 0:
            return False
        f += 2
    return True


def primes_pm1_mod8(lo: int, hi: int) -> list:
    return [p for p in range(lo | 1, hi + 1, 2) if p % 8 in (1, 7) and is_prime(p)]


def sieve_compatible(r: int, dmax: int) -> bool:
    """gcd(r mod (2^d-1), 2^d-1) == 1 for every d <= dmax (sieve_ref.cpp:79-83)."""
    from math import gcd
    for d in range(2, dmax + 1):
        M = (1 << d) - 1
        rm = r % M
        if gcd(rm if rm else M, M) != 1:
            return False
    return True


def sieve_config(seed: int = 1, dmax: int = 20):
    rng = np.random.default_rng(seed)
    cands = [p for p in primes_pm1_mod8(40000, 50000) if sieve_compatible(p, dmax)]
    r = int(cands[int(rng.integers(len(cands)))])
    return {"r": r, "dmax": dmax, "smax": r // 2}


def squaring_config(seed: int = 1, nstates: int = 256, k: int = 4096, near: int = 1_000_000):
    rng = np.random.default_rng(seed)
    cands = primes_pm1_mod8(near - 2000, near + 2000)
    r = int(cands[int(rng.integers(len(cands)))])
    s = rng.integers(3, r // 2 + 1, size=nstates, dtype=np.int64).astype(np.uint64)
    return {"r": r, "s": s, "k": k}


def splitmix64(seed: int, n: int) -> np.ndarray:
    """n outputs of SplitMix64 from `seed` (vectorised)."""
    idx = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + idx * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def random_bits(bits: int, seed: int) -> np.ndarray:
    w = splitmix64(seed, (bits + 63) >> 6)
    if bits & 63:
        w[-1] &= np.uint64((1 << (bits & 63)) - 1)
    return w


def mul_config(seed: int = 1, npairs: int = 64, lo: float = 16.0, hi: float = 27.0):
    rng = np.random.default_rng(seed)
    U = rng.uniform(lo, hi, size=(npairs, 2))
    sizes = [(int(2 ** u), int(2 ** v)) for u, v in U]
    return {"sizes": sizes, "seed": seed}
