"""Host-side GF(2^64) helpers (x^64 + x^4 + x^3 + x + 1) used for argument
checks such as CantorBasis.verify (gf2_cantor_engine.h:105-121)."""


def gf64_mul_host(a: int, b: int) -> int:
    r = 0
    while b:
        if b & 1:
            r ^= a
        hi = a >> 63
        a = ((a << 1) & 0xFFFFFFFFFFFFFFFF) ^ (0x1B if hi else 0)
        b >>= 1
    return r
