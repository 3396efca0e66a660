// trin_ctx.cu -- the TrinGPU context of the reference
// (gf2_trinomial_cuda.h:87-178) behind the C ABI: F = x^(2^k) mod T (dA),
// the running product ACC (dACC), a 2r-bit product buffer (dT0) and an FFT
// plan sized for r-bit x r-bit products.
#include "gf2e_internal.cuh"
#include "wrapmul.cuh"

#include <cstdlib>

namespace gf2e {
int trin_reduce(const u64 *P, size_t pw, u64 L, u64 *out, u64 r, u64 s, cudaStream_t st);
int trin_square(const u64 *in, u64 *out, u64 r, u64 s, cudaStream_t st);
int trin_set_const(u64 *states, size_t stride, int nstates, u64 r, u64 w0, cudaStream_t st);
int mul(const gf2e_fft_plan *plan, const u64 *a, u64 abits, const u64 *b, u64 bbits,
        u64 *out, u64 *fa, u64 *fb, cudaStream_t st);
int mul_fft_m(u64 abits, u64 bbits);
gf2e_fft_plan *cached_plan(int m);
int frobenius_states(u64 *a, u64 *b, size_t stride, int nstates, u64 r, const u64 *s_dev,
                     u64 k, cudaStream_t st, u64 s_uniform);
}  // namespace gf2e

namespace {
__global__ void k_xor_word0(u64 *p, u64 v) {
    if (blockIdx.x == 0 && threadIdx.x == 0) p[0] ^= v;
}
}  // namespace

struct gf2e_trin {
    u64 r = 0, s = 0;
    size_t nw = 0;
    int m = 0;                            // transform size the products run at
    int m_full = 0;                       // 2^m_full >= 2 ceil(r/32) - 1 (TrinGPU::m)
    gf2e_fft_plan *plan = nullptr;
    u64 *dA = nullptr, *dACC = nullptr, *dT0 = nullptr, *dT1 = nullptr;
    u64 *dFA = nullptr, *dFB = nullptr;
    bool wrap = false;                    // r-bit products one size smaller (wrapmul.cu)
    gf2e::WrapMul wm;
    u64 *dWS = nullptr;
};

namespace {
int ctx_mul(gf2e_trin *c, const u64 *x, const u64 *y, cudaStream_t st) {
    if (c->wrap)
        return gf2e::mul_wrapped(c->wm, x, c->r, y, c->r, c->dT0, c->dFA, c->dFB, c->dWS, st);
    return gf2e::mul(c->plan, x, c->r, y, c->r, c->dT0, c->dFA, c->dFB, st);
}
}  // namespace

extern "C" {

int gf2e_trin_create(uint64_t r, gf2e_trin **out) {
    if (!out) return gf2e::invalid("null context pointer");
    if (r < 5 || !(r & 1)) return gf2e::invalid("r must be odd and >= 5");
    gf2e_trin *c = new gf2e_trin;
    c->r = r;
    c->nw = (size_t)((r + 63) >> 6);
    c->m = c->m_full = gf2e::mul_fft_m(r, r);
    c->wrap = !getenv("GF2E_NO_WRAP") && gf2e::wrap_mul_plan(r, r, c->wm) &&
              gf2e::wrap_mul_plans(c->wm);
    if (c->wrap) c->m = c->wm.mb;
    c->plan = gf2e::cached_plan(c->m);
    if (!c->plan) {
        const int m = c->m;
        delete c;
        return gf2e::invalid("FFT plan for m=%d failed", m);
    }
    // the transform buffers and dT1 have the reference's sizes (2^m_full
    // points, 2 nw words), so callers may use them as TrinGPU's dFA, dFB and
    // dT1; wrapped products use the first 2^m points
    size_t n = (size_t)1 << c->m_full;
    // dA has an even word count (the two-squaring pass stores word pairs)
    cudaError_t e = cudaMalloc(&c->dA, (c->nw + (c->nw & 1)) * 8);
    if (e == cudaSuccess) e = cudaMalloc(&c->dACC, c->nw * 8);
    if (e == cudaSuccess) e = cudaMalloc(&c->dT0, (2 * c->nw + 2) * 8);
    if (e == cudaSuccess) e = cudaMalloc(&c->dT1, (2 * c->nw + 2) * 8);
    if (e == cudaSuccess) e = cudaMalloc(&c->dFA, n * 8);
    if (e == cudaSuccess) e = cudaMalloc(&c->dFB, n * 8);
    if (e == cudaSuccess && c->wrap) e = cudaMalloc(&c->dWS, c->wm.per * 8);
    if (e != cudaSuccess) {
        gf2e_trin_destroy(c);
        return gf2e::cuda_status(e, "trin context allocation");
    }
    *out = c;
    return GF2E_OK;
}

int gf2e_trin_destroy(gf2e_trin *c) {
    if (!c) return GF2E_OK;
    cudaFree(c->dA); cudaFree(c->dACC); cudaFree(c->dT0); cudaFree(c->dT1);
    cudaFree(c->dFA); cudaFree(c->dFB); cudaFree(c->dWS);
    delete c;
    return GF2E_OK;
}

int gf2e_trin_set_s(gf2e_trin *c, uint64_t s) {
    if (!c) return gf2e::invalid("null context");
    if (!(s >= 1 && 2 * s < c->r)) return gf2e::invalid("need 1 <= s <= (r-1)/2");
    c->s = s;
    return GF2E_OK;
}

int gf2e_trin_buffers(gf2e_trin *c, uint64_t **dA, uint64_t **dACC, uint64_t **dT0,
                      size_t *nw, int *m) {
    if (!c) return gf2e::invalid("null context");
    if (dA) *dA = c->dA;
    if (dACC) *dACC = c->dACC;
    if (dT0) *dT0 = c->dT0;
    if (nw) *nw = c->nw;
    if (m) *m = c->m;
    return GF2E_OK;
}

int gf2e_trin_scratch(gf2e_trin *c, uint64_t **dT1, uint64_t **dFA, uint64_t **dFB,
                      int *m_full) {
    if (!c) return gf2e::invalid("null context");
    if (dT1) *dT1 = c->dT1;
    if (dFA) *dFA = c->dFA;
    if (dFB) *dFB = c->dFB;
    if (m_full) *m_full = c->m_full;
    return GF2E_OK;
}

int gf2e_trin_reset_A(gf2e_trin *c, void *stream) {
    if (!c) return gf2e::invalid("null context");
    return gf2e::trin_set_const(c->dA, c->nw, 1, c->r, 2, (cudaStream_t)stream);
}

int gf2e_trin_reset_acc(gf2e_trin *c, void *stream) {
    if (!c) return gf2e::invalid("null context");
    return gf2e::trin_set_const(c->dACC, c->nw, 1, c->r, 1, (cudaStream_t)stream);
}

int gf2e_trin_square_A(gf2e_trin *c, void *stream) {
    if (!c || !c->s) return gf2e::invalid("context without s");
    cudaStream_t st = (cudaStream_t)stream;
    GF2E_TRY(gf2e::trin_square(c->dA, c->dT1, c->r, c->s, st));
    cudaError_t e = cudaMemcpyAsync(c->dA, c->dT1, c->nw * 8, cudaMemcpyDeviceToDevice, st);
    return gf2e::cuda_status(e, "square_A copy");
}

int gf2e_trin_square_A_k(gf2e_trin *c, uint64_t k, void *stream) {
    if (!c || !c->s) return gf2e::invalid("context without s");
    return gf2e::frobenius_states(c->dA, c->dT1, c->nw + (c->nw & 1), 1, c->r, nullptr, k,
                                  (cudaStream_t)stream, c->s);
}

int gf2e_trin_mul_dev(gf2e_trin *c, const uint64_t *x, const uint64_t *y, void *stream) {
    if (!c || !x || !y) return gf2e::invalid("null argument");
    return ctx_mul(c, x, y, (cudaStream_t)stream);
}

int gf2e_trin_reduce_T0(gf2e_trin *c, uint64_t *dst, uint64_t L, void *stream) {
    if (!c || !dst || !c->s) return gf2e::invalid("context without s / null dst");
    if (L > 2 * c->r - 1) return gf2e::invalid("L > 2r-1");
    return gf2e::trin_reduce(c->dT0, (size_t)((L + 63) >> 6), L, dst, c->r, c->s,
                             (cudaStream_t)stream);
}

int gf2e_trin_accumulate(gf2e_trin *c, void *stream) {
    if (!c || !c->s) return gf2e::invalid("context without s");
    cudaStream_t st = (cudaStream_t)stream;
    k_xor_word0<<<1, 32, 0, st>>>(c->dA, 2);                  // F + x
    GF2E_CHECK_LAUNCH("k_xor_word0");
    GF2E_TRY(ctx_mul(c, c->dACC, c->dA, st));
    k_xor_word0<<<1, 32, 0, st>>>(c->dA, 2);                  // restore F
    GF2E_CHECK_LAUNCH("k_xor_word0");
    return gf2e::trin_reduce(c->dT0, (size_t)((2 * c->r - 1 + 63) >> 6), 2 * c->r - 1, c->dACC,
                             c->r, c->s, st);
}

}  // extern "C"
