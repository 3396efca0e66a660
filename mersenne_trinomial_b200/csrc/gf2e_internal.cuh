// gf2e_internal.cuh -- shared device arithmetic and host error plumbing for
// libgf2e.so.  sm_100a only.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>
#include <stdio.h>
#include <stdarg.h>

#include "../../include/gf2e.h"

typedef uint64_t u64;
typedef uint32_t u32;

// ---------------------------------------------------------------------------
// host-side error state (thread-local detail string)
namespace gf2e {

void set_error(const char *fmt, ...);

inline int cuda_status(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return GF2E_OK;
    set_error("%s: %s", what, cudaGetErrorString(e));
    return GF2E_ERR_CUDA;
}

inline int invalid(const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    set_error("%s", buf);
    return GF2E_ERR_INVALID;
}

// grid size for a grid-stride kernel: multiple of the SM count, capped
int grid_for(size_t work, int threads, int ctas_per_sm = 8);
int sm_count();

// process-wide tuning in force (defaults, then environment overrides)
gf2e_tune tune_current();

}  // namespace gf2e

#define GF2E_CHECK_LAUNCH(what)                                              \
    do {                                                                     \
        cudaError_t _e = cudaGetLastError();                                 \
        if (_e != cudaSuccess) return gf2e::cuda_status(_e, what);           \
    } while (0)

#define GF2E_TRY(x)                                                          \
    do {                                                                     \
        int _st = (x);                                                       \
        if (_st != GF2E_OK) return _st;                                      \
    } while (0)

// ---------------------------------------------------------------------------
// device arithmetic
#define GF2E_DEV __device__ __forceinline__

// spread the low 16 bits of a 32-bit word to the even bit positions
// (interleave zeros); the first step is one byte permute.
GF2E_DEV u32 spread16_lo(u32 v) {
    u32 x = __byte_perm(v, 0u, 0x4140);           // [b0, 0, b1, 0]
    x = (x | (x << 4)) & 0x0F0F0F0Fu;
    x = (x | (x << 2)) & 0x33333333u;
    x = (x | (x << 1)) & 0x55555555u;
    return x;
}
GF2E_DEV u32 spread16_hi(u32 v) {
    u32 x = __byte_perm(v, 0u, 0x4342);           // [b2, 0, b3, 0]
    x = (x | (x << 4)) & 0x0F0F0F0Fu;
    x = (x | (x << 2)) & 0x33333333u;
    x = (x | (x << 1)) & 0x55555555u;
    return x;
}
// squaring of a 32-bit GF(2)[x] chunk: 64-bit result at even positions
GF2E_DEV u64 spread32(u32 v) {
    return ((u64)spread16_hi(v) << 32) | (u64)spread16_lo(v);
}

// carry-less 32x32 -> 64 product with integer multiplies on operands whose
// set bits are 4 apart: every column of a partial product then sums at most
// 8 ones, which never carries into the next column of the same residue
// class mod 4, so masking each partial product to its class recovers the
// XOR sum.
// 32 x 32 -> 64 integer product (one widening multiply)
GF2E_DEV u64 mulw32(u32 a, u32 b) {
    u64 r;
    asm("mul.wide.u32 %0, %1, %2;" : "=l"(r) : "r"(a), "r"(b));
    return r;
}
// a 32-bit operand split into its four bit classes mod 4
struct Masked {
    u32 p[4];
};
GF2E_DEV Masked mask32(u32 a) {
    Masked m;
    m.p[0] = a & 0x11111111u;
    m.p[1] = a & 0x22222222u;
    m.p[2] = a & 0x44444444u;
    m.p[3] = a & 0x88888888u;
    return m;
}
// the product from operands already split (a matrix entry or a word used
// in several products is split once)
GF2E_DEV u64 clmul_masked(const Masked &a, const Masked &b) {
    const u64 M0 = 0x1111111111111111ull;
    const u64 c0 = mulw32(a.p[0], b.p[0]) ^ mulw32(a.p[1], b.p[3]) ^ mulw32(a.p[2], b.p[2]) ^
                   mulw32(a.p[3], b.p[1]);
    const u64 c1 = mulw32(a.p[0], b.p[1]) ^ mulw32(a.p[1], b.p[0]) ^ mulw32(a.p[2], b.p[3]) ^
                   mulw32(a.p[3], b.p[2]);
    const u64 c2 = mulw32(a.p[0], b.p[2]) ^ mulw32(a.p[1], b.p[1]) ^ mulw32(a.p[2], b.p[0]) ^
                   mulw32(a.p[3], b.p[3]);
    const u64 c3 = mulw32(a.p[0], b.p[3]) ^ mulw32(a.p[1], b.p[2]) ^ mulw32(a.p[2], b.p[1]) ^
                   mulw32(a.p[3], b.p[0]);
    return (c0 & M0) ^ (c1 & (M0 << 1)) ^ (c2 & (M0 << 2)) ^ (c3 & (M0 << 3));
}
GF2E_DEV u64 clmul32(u32 a, u32 b) { return clmul_masked(mask32(a), mask32(b)); }

// GF(2^64) = GF(2)[x]/(x^64 + x^4 + x^3 + x + 1) multiply (Karatsuba over
// clmul32 and the two-step reduction by the sparse modulus).
GF2E_DEV u64 gf64_mul(u64 a, u64 b) {
    u32 a0 = (u32)a, a1 = (u32)(a >> 32), b0 = (u32)b, b1 = (u32)(b >> 32);
    u64 lo = clmul32(a0, b0);
    u64 hi = clmul32(a1, b1);
    u64 mid = clmul32(a0 ^ a1, b0 ^ b1) ^ lo ^ hi;
    lo ^= mid << 32;
    hi ^= mid >> 32;
    u64 t = lo ^ hi ^ (hi << 1) ^ (hi << 3) ^ (hi << 4);
    u64 h2 = (hi >> 63) ^ (hi >> 61) ^ (hi >> 60);
    return t ^ h2 ^ (h2 << 1) ^ (h2 << 3) ^ (h2 << 4);
}

// 64-bit funnel: bits [sh, sh+64) of the 128-bit value (hi:lo), 0 <= sh < 64
GF2E_DEV u64 funnel64(u64 lo, u64 hi, unsigned sh) {
    return sh ? ((lo >> sh) | (hi << (64 - sh))) : lo;
}

// low `n` bits set, 0 <= n <= 64
GF2E_DEV u64 low_mask(u64 n) { return n >= 64 ? ~0ull : ((1ull << n) - 1); }
