// wrapmul.cuh -- products one transform size smaller with the wrapped part
// put back (wrapmul.cu).
#pragma once

#include "gf2e_internal.cuh"

namespace gf2e {

struct WrapTerms {
    int n;
    u64 z[24];          // shifts of OA(Q), in 32-bit chunks
};

struct WrapMul {
    int mb = 0, ms = 0;                  // transform sizes: the product's, the top part's
    u64 n = 0, ns = 0, T = 0, D = 0, p = 0, q = 0;
    u64 xw = 0, nsch = 0, uw = 0, qw = 0;
    WrapTerms terms{};
    gf2e_fft_plan *big = nullptr, *small = nullptr;
    // scratch per batch element, in words: Xa, Xb, FAs, FBs, U, Q
    u64 off_xa = 0, off_xb = 0, off_fa = 0, off_fb = 0, off_u = 0, off_q = 0, per = 0;
};

// the wrapped geometry for abits x bbits products (host arithmetic only),
// false when the plain size is the better or the only choice
bool wrap_mul_plan(u64 abits, u64 bbits, WrapMul &w);
// the two transform plans of a wrapped product (on the current device)
bool wrap_mul_plans(WrapMul &w);

// after the 2^mb transform product of a and b left R (2^mb coefficients per
// batch element, stride rstride words): P = a b, ow words per element.
// scratch holds batch * w.per words.
int wrap_mul_finish(const WrapMul &w, const u64 *R, u64 rstride, const u64 *a, u64 astride,
                    const u64 *b, u64 bstride, u64 *P, u64 pstride, u64 ow, int batch,
                    u64 *scratch, cudaStream_t st);

// out = a b for one product ((abits + bbits + 63) / 64 + 1 words); fa and
// fb of 2^mb words, scratch of w.per words
int mul_wrapped(const WrapMul &w, const u64 *a, u64 abits, const u64 *b, u64 bbits, u64 *out,
                u64 *fa, u64 *fb, u64 *scratch, cudaStream_t st);

}  // namespace gf2e
