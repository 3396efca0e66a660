"""TEST INFRASTRUCTURE ONLY: ctypes front end to the CPU oracle.

The oracle (oracle/gf2_oracle.c -> oracle/liboracle.so) is the CPU
restatement of the reference algorithms that the CUDA engine is checked
against.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg import this module.  The product package never does.

`ref_*` helpers wrap the reference's own code built by oracle/build_ref.sh
into oracle/_ref/ (present only where the reference sources were available
at build time; callers must tolerate their absence).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_lib = None
_ref_cantor = None


def build() -> None:
    """Compile liboracle.so (and the reference tools when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
        L = C.CDLL(LIB_PATH)
        u64, u32, i32 = C.c_uint64, C.c_uint32, C.c_int
        L.orc_gf_mul.argtypes = [u32, u32, u64, i32]
        L.orc_gf_mul.restype = u32
        L.orc_find_primitive_poly.argtypes = [i32]
        L.orc_find_primitive_poly.restype = u64
        L.orc_is_irreducible.argtypes = [u64, i32]
        L.orc_is_irreducible.restype = i32
        L.orc_sieve.argtypes = [u64, i32, i32, u64, _u64p, i32, C.c_void_p, C.c_void_p]
        L.orc_sieve.restype = i32
        L.orc_sieve_brute.argtypes = [u64, i32, u64, _u64p]
        L.orc_sieve_brute.restype = None
        L.orc_trin_square.argtypes = [_u64p, _u64p, u64, u64]
        L.orc_trin_square.restype = i32
        L.orc_trin_square_k.argtypes = [_u64p, u64, u64, u64]
        L.orc_trin_square_k.restype = i32
        L.orc_trin_square_naive.argtypes = [_u64p, u64, u64]
        L.orc_trin_square_naive.restype = i32
        L.orc_mod_trinomial.argtypes = [_u64p, u64, u64, u64]
        L.orc_mod_trinomial.restype = None
        L.orc_naive_mul.argtypes = [_u64p, u64, _u64p, u64, _u64p]
        L.orc_naive_mul.restype = None
        L.orc_comb_mul.argtypes = [_u64p, u64, _u64p, u64, _u64p]
        L.orc_comb_mul.restype = None
        L.orc_fft_mul.argtypes = [_u64p, u64, _u64p, u64, _u64p]
        L.orc_fft_mul.restype = i32
        L.orc_fft_m_for.argtypes = [u64, u64]
        L.orc_fft_m_for.restype = i32
        L.orc_cantor_basis.argtypes = [_u64p]
        L.orc_cantor_basis.restype = i32
        L.orc_fft_twiddles.argtypes = [i32, _u64p, _u64p]
        L.orc_fft_twiddles.restype = None
        L.orc_fft_fwd.argtypes = [_u64p, i32, _u64p]
        L.orc_fft_fwd.restype = None
        L.orc_fft_inv.argtypes = [_u64p, i32, _u64p]
        L.orc_fft_inv.restype = None
        L.orc_gf64_mul.argtypes = [u64, u64]
        L.orc_gf64_mul.restype = u64
        L.orc_gf64_mul_bitref.argtypes = [u64, u64]
        L.orc_gf64_mul_bitref.restype = u64
        L.orc_residue.argtypes = [_u64p, u64, u64, i32]
        L.orc_residue.restype = u64
        L.orc_modq_mul.argtypes = [u64, u64, u64, i32]
        L.orc_modq_mul.restype = u64
        L.orc_poly_gcd.argtypes = [_u64p, C.c_size_t, _u64p, C.c_size_t, _u64p, C.c_size_t]
        L.orc_poly_gcd.restype = C.c_int64
        L.orc_factor_divides.argtypes = [u64, u64, u64, _u64p, C.c_size_t]
        L.orc_factor_divides.restype = i32
        L.orc_edf_least_enum.argtypes = [_u64p, C.c_size_t, u64]
        L.orc_edf_least_enum.restype = u64
        L.orc_scan_one.argtypes = [u64, u64, u64, u64, C.POINTER(u64), C.POINTER(u64),
                                   _u64p, _u64p, C.c_size_t, C.POINTER(C.c_int)]
        L.orc_scan_one.restype = i32
        _lib = L
    return _lib


def words(bits: int) -> int:
    return (int(bits) + 63) >> 6


def mul_out_words(abits: int, bbits: int) -> int:
    return words(abits + bbits) + 1


# ---------------------------------------------------------------- sieve
def sieve(r: int, dmax: int, smax: int, dmin: int = 2, best=None, stats=False):
    """best[s] = min key (d<<48)|mask over factors of degree dmin..dmax (sieve_ref.cpp:58-134)."""
    init = best is None
    if best is None:
        best = np.zeros(smax + 1, dtype=np.uint64)
    cls = np.zeros(64, dtype=np.uint64)
    mk = np.zeros(64, dtype=np.uint64)
    rc = lib().orc_sieve(r, dmin, dmax, smax, best, int(init),
                         cls.ctypes.data_as(C.c_void_p), mk.ctypes.data_as(C.c_void_p))
    if rc != 0:
        raise ValueError(f"oracle sieve failed rc={rc} (gcd(r, 2^d-1) != 1 at d={-rc})")
    if stats:
        return best, cls, mk
    return best


def sieve_brute(r: int, depth: int, smax: int):
    best = np.zeros(smax + 1, dtype=np.uint64)
    lib().orc_sieve_brute(r, depth, smax, best)
    return best


def cert_lines(best, skip_s2: bool = False):
    """'s d p<hex>' for every s with a factor (sieve_ref.cpp:163-169, 205-206)."""
    out = []
    b = np.asarray(best)
    idx = np.nonzero(b != np.uint64(0xFFFFFFFFFFFFFFFF))[0]
    for s in idx:
        s = int(s)
        if s == 0 or (skip_s2 and s == 2):
            continue
        k = int(b[s])
        out.append(f"{s} {k >> 48} p{k & 0xFFFFFFFFFFFF:x}")
    return out


# ------------------------------------------------------------- trinomial
def x_state(r: int) -> np.ndarray:
    st = np.zeros(words(r), dtype=np.uint64)
    st[0] = 2
    return st


def trin_square_k(state: np.ndarray, r: int, s: int, k: int) -> np.ndarray:
    st = np.ascontiguousarray(state, dtype=np.uint64).copy()
    if lib().orc_trin_square_k(st, r, s, k) != 0:
        raise ValueError("need 1 <= s <= (r-1)/2")
    return st


def trin_square_naive(state: np.ndarray, r: int, s: int) -> np.ndarray:
    st = np.ascontiguousarray(state, dtype=np.uint64).copy()
    if lib().orc_trin_square_naive(st, r, s) != 0:
        raise ValueError("need 1 <= s <= (r-1)/2")
    return st


def mod_trinomial(v: np.ndarray, nbits: int, r: int, s: int) -> np.ndarray:
    """naive bit-serial reduction mod x^r+x^s+1 (gf2_trinomial_cuda.h:182-190)."""
    v = np.ascontiguousarray(v, dtype=np.uint64).copy()
    lib().orc_mod_trinomial(v, nbits, r, s)
    return v[: words(r)].copy()


# ------------------------------------------------------------- multiply
def _bits_arr(a, bits):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    if a.size < words(bits):
        a = np.concatenate([a, np.zeros(words(bits) - a.size, dtype=np.uint64)])
    return a


def fft_mul(a, abits, b, bbits):
    out = np.zeros(mul_out_words(abits, bbits), dtype=np.uint64)
    rc = lib().orc_fft_mul(_bits_arr(a, abits), abits, _bits_arr(b, bbits), bbits, out)
    if rc != 0:
        raise ValueError(f"oracle fft_mul rc={rc}")
    return out


def comb_mul(a, abits, b, bbits):
    out = np.zeros(mul_out_words(abits, bbits), dtype=np.uint64)
    lib().orc_comb_mul(_bits_arr(a, abits), abits, _bits_arr(b, bbits), bbits, out)
    return out


def naive_mul(a, abits, b, bbits):
    out = np.zeros(mul_out_words(abits, bbits), dtype=np.uint64)
    lib().orc_naive_mul(_bits_arr(a, abits), abits, _bits_arr(b, bbits), bbits, out)
    return out


def cantor_basis():
    b = np.zeros(64, dtype=np.uint64)
    n = lib().orc_cantor_basis(b)
    return b[:n].copy()


def fft_twiddles(m: int):
    b = np.zeros(64, dtype=np.uint64)
    lib().orc_cantor_basis(b)
    W = np.zeros(max(1, 1 << (m - 1)), dtype=np.uint64)
    lib().orc_fft_twiddles(m, b, W)
    return W


def fft_fwd(f, m):
    f = np.ascontiguousarray(f, dtype=np.uint64).copy()
    lib().orc_fft_fwd(f, m, fft_twiddles(m))
    return f


def fft_inv(f, m):
    f = np.ascontiguousarray(f, dtype=np.uint64).copy()
    lib().orc_fft_inv(f, m, fft_twiddles(m))
    return f


def residue(a, abits, q, d):
    return int(lib().orc_residue(_bits_arr(a, abits), abits, q, d))


def modq_mul(a, b, q, d):
    return int(lib().orc_modq_mul(a, b, q, d))


# ------------------------------------------------------------- gcd / verify
def poly_gcd(a, b):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    cap = max(a.size, b.size) + 1
    g = np.zeros(cap, dtype=np.uint64)
    d = lib().orc_poly_gcd(a, a.size, b, b.size, g, cap)
    return int(d), g


def hex_to_words(h: str) -> np.ndarray:
    v = int(h, 16)
    n = max(1, (v.bit_length() + 63) // 64)
    return np.array([(v >> (64 * i)) & 0xFFFFFFFFFFFFFFFF for i in range(n)], dtype=np.uint64)


def factor_divides(r: int, s: int, d: int, hexmask: str) -> int:
    """check-ntl.c:17-58 restated: 1 divides, 0 does not, -1 degree mismatch."""
    f = hex_to_words(hexmask)
    return int(lib().orc_factor_divides(r, s, d, f, f.size))


def verify_cert_lines(r: int, lines) -> int:
    """Number of lines that fail the divisibility check (0 = all good)."""
    bad = 0
    for ln in lines:
        parts = ln.split()
        if len(parts) < 3 or parts[1] in ("u", "primitive"):
            continue
        s, d, p = int(parts[0]), int(parts[1]), parts[2]
        if not p.startswith("p") or factor_divides(r, s, d, p[1:]) != 1:
            bad += 1
    return bad


def scan_one(r: int, s: int, k0: int, maxd: int):
    """trinomial_scan.cu:393-421: (status, d, gdeg, g_hex, mask_hex)."""
    cap = words(r + 1) + 1
    g = np.zeros(cap, dtype=np.uint64)
    mask = np.zeros(cap, dtype=np.uint64)
    d = C.c_uint64(0)
    gd = C.c_uint64(0)
    ok = C.c_int(0)
    st = lib().orc_scan_one(r, s, k0, maxd, C.byref(d), C.byref(gd), g, mask, cap, C.byref(ok))
    return int(st), int(d.value), int(gd.value), words_hex(g), (words_hex(mask) if ok.value else None)


def words_hex(v) -> str:
    x = 0
    for i, w in enumerate(np.asarray(v, dtype=np.uint64).tolist()):
        x |= int(w) << (64 * i)
    return format(x, "x")


def edf_least_enum(g, target: int) -> int:
    g = np.ascontiguousarray(g, dtype=np.uint64)
    return int(lib().orc_edf_least_enum(g, g.size, target))


# ------------------------------------------------------------- reference (oracle/_ref)
def ref_available(name: str) -> bool:
    return os.path.exists(os.path.join(REF_DIR, name))


def ref_cantor():
    global _ref_cantor
    if _ref_cantor is None:
        p = os.path.join(REF_DIR, "libref_cantor.so")
        if not os.path.exists(p):
            return None
        L = C.CDLL(p)
        L.ref_fft_mul.argtypes = [_u64p, C.c_uint64, _u64p, C.c_uint64, _u64p]
        L.ref_fft_mul.restype = C.c_int
        L.ref_fft_fwd.argtypes = [_u64p, C.c_int]
        L.ref_fft_inv.argtypes = [_u64p, C.c_int]
        L.ref_basis.argtypes = [_u64p]
        L.ref_basis.restype = C.c_int
        L.ref_twiddles.argtypes = [C.c_int, _u64p]
        L.ref_twiddles.restype = C.c_int
        L.ref_gf64_mul.argtypes = [C.c_uint64, C.c_uint64]
        L.ref_gf64_mul.restype = C.c_uint64
        _ref_cantor = L
    return _ref_cantor
