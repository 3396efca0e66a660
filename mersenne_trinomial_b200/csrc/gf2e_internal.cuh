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
GF2E_DEV u64 clmul32(u32 a, u32 b) {
    const u32 m0 = 0x11111111u, m1 = 0x22222222u, m2 = 0x44444444u,
              m3 = 0x88888888u;
    u64 a0 = a & m0, a1 = a & m1, a2 = a & m2, a3 = a & m3;
    u64 b0 = b & m0, b1 = b & m1, b2 = b & m2, b3 = b & m3;
    const u64 M0 = 0x1111111111111111ull;
    u64 c0 = (a0 * b0) ^ (a1 * b3) ^ (a2 * b2) ^ (a3 * b1);
    u64 c1 = (a0 * b1) ^ (a1 * b0) ^ (a2 * b3) ^ (a3 * b2);
    u64 c2 = (a0 * b2) ^ (a1 * b1) ^ (a2 * b0) ^ (a3 * b3);
    u64 c3 = (a0 * b3) ^ (a1 * b2) ^ (a2 * b1) ^ (a3 * b0);
    return (c0 & M0) ^ (c1 & (M0 << 1)) ^ (c2 & (M0 << 2)) ^ (c3 & (M0 << 3));
}

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
