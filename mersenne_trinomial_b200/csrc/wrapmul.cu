// wrapmul.cu -- products one transform size smaller: a GF(2)[x] product
// whose chunk count exceeds a power of two by a little (r = 136279841 needs
// 8,517,489 coefficients against 2^23 = 8,388,608) is taken with the 2^m
// transform anyway and the wrapped part is put back.
//
// With chunks of 32 bits, A(y) B(y) (y = x^32) has coefficients c_k, k < 2^m
// + delta.  The transform of size 2^m evaluates on a subspace whose
// vanishing polynomial is Z(y) = y^(2^m) + Zlow(y), Zlow = sum of y^(2^i)
// over the i < m with i & m == i (the Cantor basis' subspace polynomial), so
// the transform product returns R = A B mod Z and
//     A B = R + Q Z = R + Q Zlow + Q y^(2^m),    Q = the c_k with k >= 2^m.
// Zlow's coefficients are 1, so in bits (x^32 = y)
//     a b = OA(R) + sum over z of OA(Q) x^(32 z) + OA(Q) x^T,   T = 32 * 2^m,
// OA the overlap-add of 64-bit coefficients at 32-bit steps.  OA(Q) is the
// product's top part floor(a b / x^T) without the high half of c_(2^m - 1)
// (which lies at bits >= T): floor(a b / x^T) = floor(a_hi b_hi / x^(D-1))
// with a_hi, b_hi the top D = |a| + |b| - 1 - T bits of a and b, a product
// 1/64 the size at r = 136279841.  Exactness needs delta < 2^(m-1) (Q Zlow
// stays below 2^m); plans use it for delta <= 2^(m-2), where the two
// products together still cost at most 3/4 of the plain 2^(m+1) one.
#include "gf2e_internal.cuh"
#include "wrapmul.cuh"

#include <algorithm>
#include <vector>

namespace gf2e {
int fft_fwd_packed_batch(const gf2e_fft_plan *plan, u64 *f, u64 fstride, const u32 *src32,
                         u64 sstride32, u64 nchunks, u64 xor0, int batch, cudaStream_t st);
int fft_run_batch(const gf2e_fft_plan *plan, bool forward, u64 *f, u64 fstride, int batch,
                  cudaStream_t st);
int overlap_add_batch(const u64 *F, u64 fstride, u64 nchunks, u64 *out, u64 ostride, u64 ow,
                      int batch, cudaStream_t st);
gf2e_fft_plan *cached_plan(int m);
int mul_fft_m(u64 abits, u64 bbits);
int fft_fwd_packed(const gf2e_fft_plan *plan, u64 *f, const u32 *src32, u64 nchunks,
                   cudaStream_t st);
int fft_run(const gf2e_fft_plan *plan, bool forward, u64 *f, cudaStream_t st);
int pointwise(u64 *fa, const u64 *fb, u64 n, cudaStream_t st);
}  // namespace gf2e

namespace {

// dst[w] = bits [p + 64 w, p + 64 w + 64) of src, zero from bit nbits of dst
__global__ void k_extract_bits(const u64 *__restrict__ src, u64 sstride, u64 p, u64 nbits,
                               u64 *__restrict__ dst, u64 dstride, u64 dw) {
    src += (u64)blockIdx.y * sstride;
    dst += (u64)blockIdx.y * dstride;
    for (u64 w = (u64)blockIdx.x * blockDim.x + threadIdx.x; w < dw;
         w += (u64)gridDim.x * blockDim.x) {
        const u64 b = 64 * w;
        u64 v = 0;
        if (b < nbits) {
            const u64 pos = p + b, i = pos >> 6;
            const unsigned sh = (unsigned)(pos & 63);
            const u64 lo = src[i];
            v = sh ? (lo >> sh) : lo;
            if (sh && b + 64 - sh < nbits) v |= src[i + 1] << (64 - sh);
            if (nbits - b < 64) v &= (1ull << (nbits - b)) - 1;
        }
        dst[w] = v;
    }
}

// fa *= fb pointwise, batched with strides
__global__ void k_pointwise_batch(u64 *__restrict__ fa, const u64 *__restrict__ fb, u64 n,
                                  u64 stride) {
    fa += (u64)blockIdx.y * stride;
    fb += (u64)blockIdx.y * stride;
    for (u64 k = (u64)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (u64)gridDim.x * blockDim.x)
        fa[k] = gf64_mul(fa[k], fb[k]);
}

// OA(Q)[w] = bits [D - 1 + 64 w, ...) of U (the product a_hi b_hi), and the
// high half of R's last coefficient XORed into word 0
__global__ void k_wrap_q(const u64 *__restrict__ U, u64 ustride, u64 uw, u64 shift, u64 qbits,
                         const u64 *__restrict__ R, u64 rstride, u64 rlast,
                         u64 *__restrict__ Qo, u64 qstride, u64 qw) {
    U += (u64)blockIdx.y * ustride;
    Qo += (u64)blockIdx.y * qstride;
    for (u64 w = (u64)blockIdx.x * blockDim.x + threadIdx.x; w < qw;
         w += (u64)gridDim.x * blockDim.x) {
        const u64 b = 64 * w;
        u64 v = 0;
        if (b < qbits) {
            const u64 pos = shift + b, i = pos >> 6;
            const unsigned sh = (unsigned)(pos & 63);
            const u64 lo = i < uw ? U[i] : 0, hi = i + 1 < uw ? U[i + 1] : 0;
            v = sh ? ((lo >> sh) | (hi << (64 - sh))) : lo;
            if (qbits - b < 64) v &= (1ull << (qbits - b)) - 1;
        }
        if (w == 0) v ^= R[(u64)blockIdx.y * rstride + rlast] >> 32;
        Qo[w] = v;
    }
}

// P[w] ^= sum over the shifts z of OA(Q) placed at bit 32 z
__global__ void k_wrap_fix(u64 *__restrict__ P, u64 pstride, u64 ow, const u64 *__restrict__ Q,
                           u64 qstride, u64 qw, const gf2e::WrapTerms t) {
    P += (u64)blockIdx.y * pstride;
    Q += (u64)blockIdx.y * qstride;
    for (u64 w = (u64)blockIdx.x * blockDim.x + threadIdx.x; w < ow;
         w += (u64)gridDim.x * blockDim.x) {
        u64 v = 0;
        for (int k = 0; k < t.n; k++) {
            // bit 64 w of P takes bit 64 w - 32 z of OA(Q)
            const long long off = (long long)(64 * w) - (long long)(32 * t.z[k]);
            if (off <= -64 || off >= (long long)(64 * qw)) continue;
            if (off >= 0) {
                const u64 i = (u64)off >> 6;
                if (off & 63) {                          // a 32-bit offset
                    v ^= Q[i] >> 32;
                    if (i + 1 < qw) v ^= Q[i + 1] << 32;
                } else {
                    v ^= Q[i];
                }
            } else {                                     // off = -32
                v ^= Q[0] << 32;
            }
        }
        if (v) P[w] ^= v;
    }
}

}  // namespace

namespace gf2e {

// a wrapped plan for abits x bbits products, or false when the plain
// transform size is the better (or only) choice
bool wrap_mul_plan(u64 abits, u64 bbits, WrapMul &w) {
    const int m = mul_fft_m(abits, bbits);
    if (m < 12) return false;
    const int mb = m - 1;
    const u64 n = (u64)1 << mb;
    const u64 ca = (abits + 31) >> 5, cb = (bbits + 31) >> 5;
    if (ca > n || cb > n) return false;
    const u64 count = ca + cb - 1;
    if (count <= n || count - n > (n >> 2)) return false;
    const u64 T = 32 * n;
    if (abits + bbits - 1 < T + 64) return false;
    w.mb = mb;
    w.n = n;
    w.T = T;
    w.D = abits + bbits - 1 - T;
    w.p = T - bbits + 1;
    w.q = T - abits + 1;
    w.xw = (w.D + 63) / 64;
    w.nsch = (w.D + 31) / 32;
    w.ms = mul_fft_m(w.D, w.D);
    w.ns = (u64)1 << w.ms;
    w.uw = (2 * w.D - 1 + 63) / 64;
    w.qw = w.xw;
    w.terms.n = 0;
    for (int i = 0; i < mb; i++)
        if ((i & mb) == i) w.terms.z[w.terms.n++] = (u64)1 << i;
    w.terms.z[w.terms.n++] = n;
    auto even = [](u64 v) { return (v + 1) & ~(u64)1; };
    w.off_xa = 0;
    w.off_xb = w.off_xa + even(w.xw);
    w.off_fa = w.off_xb + even(w.xw);
    w.off_fb = w.off_fa + w.ns;
    w.off_u = w.off_fb + w.ns;
    w.off_q = w.off_u + even(w.uw);
    w.per = w.off_q + even(w.qw);
    return true;
}

bool wrap_mul_plans(WrapMul &w) {
    w.big = cached_plan(w.mb);
    w.small = cached_plan(w.ms);
    return w.big && w.small;
}

// After the 2^mb transform product of a and b left R (2^mb coefficients per
// batch element, stride rstride) in place: P = a b (ow words per element)
int wrap_mul_finish(const WrapMul &w, const u64 *R, u64 rstride, const u64 *a, u64 astride,
                    const u64 *b, u64 bstride, u64 *P, u64 pstride, u64 ow, int batch,
                    u64 *scratch, cudaStream_t st) {
    const u64 S = w.per;
    u64 *Xa = scratch + w.off_xa, *Xb = scratch + w.off_xb, *FAs = scratch + w.off_fa,
        *FBs = scratch + w.off_fb, *U = scratch + w.off_u, *Q = scratch + w.off_q;
    const unsigned nb = (unsigned)batch;
    GF2E_TRY(overlap_add_batch(R, rstride, w.n, P, pstride, ow, batch, st));
    k_extract_bits<<<dim3(grid_for(w.xw, 256, 4), nb), 256, 0, st>>>(a, astride, w.p, w.D, Xa,
                                                                        S, w.xw);
    GF2E_CHECK_LAUNCH("k_extract_bits");
    k_extract_bits<<<dim3(grid_for(w.xw, 256, 4), nb), 256, 0, st>>>(b, bstride, w.q, w.D, Xb,
                                                                        S, w.xw);
    GF2E_CHECK_LAUNCH("k_extract_bits");
    GF2E_TRY(fft_fwd_packed_batch(w.small, FAs, S, reinterpret_cast<const u32 *>(Xa), 2 * S,
                                  w.nsch, 0, batch, st));
    GF2E_TRY(fft_fwd_packed_batch(w.small, FBs, S, reinterpret_cast<const u32 *>(Xb), 2 * S,
                                  w.nsch, 0, batch, st));
    k_pointwise_batch<<<dim3(grid_for(w.ns, 256, 4), nb), 256, 0, st>>>(FAs, FBs, w.ns, S);
    GF2E_CHECK_LAUNCH("k_pointwise_batch");
    GF2E_TRY(fft_run_batch(w.small, false, FAs, S, batch, st));
    GF2E_TRY(overlap_add_batch(FAs, S, 2 * w.nsch - 1, U, S, w.uw, batch, st));
    k_wrap_q<<<dim3(grid_for(w.qw, 256, 4), nb), 256, 0, st>>>(U, S, w.uw, w.D - 1, w.D, R,
                                                                  rstride, w.n - 1, Q, S, w.qw);
    GF2E_CHECK_LAUNCH("k_wrap_q");
    k_wrap_fix<<<dim3(grid_for(ow, 256, 8), nb), 256, 0, st>>>(P, pstride, ow, Q, S, w.qw,
                                                                  w.terms);
    GF2E_CHECK_LAUNCH("k_wrap_fix");
    return GF2E_OK;
}

// one product out = a b (((abits + bbits + 63) >> 6) + 1 words) through the
// wrapped plan; fa and fb hold 2^mb words each, scratch w.per words
int mul_wrapped(const WrapMul &w, const u64 *a, u64 abits, const u64 *b, u64 bbits, u64 *out,
                u64 *fa, u64 *fb, u64 *scratch, cudaStream_t st) {
    const u64 ca = (abits + 31) >> 5, cb = (bbits + 31) >> 5;
    GF2E_TRY(fft_fwd_packed(w.big, fa, reinterpret_cast<const u32 *>(a), ca, st));
    if (b == a && bbits == abits) {
        GF2E_TRY(pointwise(fa, fa, w.n, st));
    } else {
        GF2E_TRY(fft_fwd_packed(w.big, fb, reinterpret_cast<const u32 *>(b), cb, st));
        GF2E_TRY(pointwise(fa, fb, w.n, st));
    }
    GF2E_TRY(fft_run(w.big, false, fa, st));
    const u64 ow = ((abits + bbits + 63) >> 6) + 1;
    return wrap_mul_finish(w, fa, 0, a, 0, b, 0, out, 0, ow, 1, scratch, st);
}

}  // namespace gf2e
