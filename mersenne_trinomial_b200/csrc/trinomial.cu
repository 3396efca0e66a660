// trinomial.cu -- arithmetic in GF(2)[x]/(x^r + x^s + 1): single-pass
// squaring (batched over many s), fold reduction of a product, and state
// initialisation.
//
// Squaring, derived for odd r and 1 <= s, 2s < r.  Split the input at
// h = (r+1)/2: in = A_lo + x^h A_hi.  Then
//     in^2 = A_lo^2 + x^(r+1) A_hi^2,   x^(r+1) = x^(s+1) + x  (mod T).
// A_lo^2 has degree <= r-1 and needs no reduction.  With S = A_hi^2 (the
// bit-spread of A_hi, degree <= r-3):
//     x*S                      degree <= r-2
//     x^(s+1)*S = Y_lo + x^r Y_hi,  Y_hi = S >> (r-s-1),  deg Y_hi <= s-2
//     x^r Y_hi = Y_hi + x^s Y_hi     (degree <= 2s-2 < r, no further fold)
// so every output word is the XOR of five 64-bit windows:
//     spread(A_lo)[w] ^ S<<1 ^ (S<<(s+1) mod x^r) ^ S>>(r-s-1)
//                     ^ (S>>(r-s-1))<<s.
// A 64-bit window of S starting at bit p is the spread of 32 bits of A_hi
// starting at ceil(p/2) (shifted left one place when p is odd), i.e. ONE
// funnel-shifted 32-bit read of the input and one spread per window.  The
// last two windows are zero outside the first ~2s/64 words and are skipped
// there.  This is the same identity the reference's fused squaring
// evaluates as five clipped windows of the virtual spread
// (tsfactor.cu:128-186); the output is bit-identical.
#include "gf2e_internal.cuh"

#include <algorithm>

namespace {

// in bits [P, P+32) of a state held as n32 32-bit words (zero beyond)
GF2E_DEV u32 in_bits32(const u32 *__restrict__ in32, size_t n32, u64 P) {
    size_t i = (size_t)(P >> 5);
    unsigned sh = (unsigned)(P & 31);
    u32 lo = (i < n32) ? __ldg(in32 + i) : 0u;
    u32 hi = (i + 1 < n32) ? __ldg(in32 + i + 1) : 0u;
    return __funnelshift_r(lo, hi, sh);
}

// S bits [p, p+64), S = spread(A_hi), A_hi = in >> h; p may be negative
GF2E_DEV u64 s_window(const u32 *__restrict__ in32, size_t n32, u64 h, int64_t p) {
    int64_t j = (p + 1) >> 1;                     // first A_hi index used
    u32 a;
    if (j >= 0)
        a = in_bits32(in32, n32, h + (u64)j);
    else if (j > -32)
        a = in_bits32(in32, n32, h) << (unsigned)(-j);
    else
        a = 0;
    u64 v = spread32(a);
    return (p & 1) ? (v << 1) : v;
}

// one output word of in^2 mod T
GF2E_DEV u64 square_word(const u32 *__restrict__ in32, size_t n32, u64 r, u64 h,
                         u64 s, size_t w) {
    const u64 b = (u64)w << 6;
    u64 v = 0;
    if (32 * (u64)w < h) {                        // spread(A_lo)
        u32 a = __ldg(in32 + w);
        u64 valid = h - 32 * (u64)w;
        if (valid < 32) a &= (1u << valid) - 1u;
        v = spread32(a);
    }
    v ^= s_window(in32, n32, h, (int64_t)b - 1);                   // S<<1
    u64 t3 = s_window(in32, n32, h, (int64_t)b - (int64_t)s - 1);  // S<<(s+1)
    if (b + 64 > r) t3 &= low_mask(r - b);
    v ^= t3;
    if (b + 1 < s)                                                   // S>>(r-s-1)
        v ^= s_window(in32, n32, h, (int64_t)(b + r - s - 1));
    if (b + 64 > s && b + 1 < 2 * s) {                               // (..)<<s
        u64 t5 = s_window(in32, n32, h, (int64_t)(b + r - 2 * s - 1));
        if (b < s) t5 &= ~low_mask(s - b);
        v ^= t5;
    }
    return v;
}

constexpr int WPT = 8;          // output words per thread on the fast path

// interleave two 16-bit values (low halves of e, o): bit 2i <- e_i,
// bit 2i+1 <- o_i.  One byte permute places [e.b0, o.b0, e.b1, o.b1], then
// three delta swaps finish the outer perfect shuffle inside each 16 bits.
// In each swap the masked bits t and t << k are disjoint, so t ^ (t << k)
// is t * (2^k + 1): one integer multiply (FMA pipe) instead of a shift and
// an XOR (ALU pipe, the busier one in this kernel).
GF2E_DEV u32 shuffle16(u32 x) {
    u32 t = (x ^ (x >> 4)) & 0x00F000F0u;
    x ^= t * 17u;
    t = (x ^ (x >> 2)) & 0x0C0C0C0Cu;
    x ^= t * 5u;
    t = (x ^ (x >> 1)) & 0x22222222u;
    x ^= t * 3u;
    return x;
}
// spread(e) ^ (spread(o) << 1) as one 64-bit word
GF2E_DEV u64 interleave32(u32 e, u32 o) {
    u32 lo = shuffle16(__byte_perm(e, o, 0x5140));
    u32 hi = shuffle16(__byte_perm(e, o, 0x7362));
    return ((u64)hi << 32) | lo;
}

// Batched squaring: blockIdx.y = state; each warp writes tiles of 32 WPT
// words, lane l the words w0 + l + 32 q.
//
// Every window is a spread of 32 input bits placed on the even bit
// positions (window offset even) or on the odd ones (offset odd), and the
// spread is linear over XOR.  So a clean group XORs the 32-bit inputs of
// all even windows into E and of all odd windows into O and writes
//     out = spread(E) ^ (spread(O) << 1):
// two spreads per output word however many windows are active.  Parities:
// spread(A_lo) and the last window are even, S<<1 is odd, the two middle
// windows are odd/even or even/odd with the parity of s.
// Warp tiles away from every window boundary take this path (32-bit index
// arithmetic, hoisted offsets, no clipping); the few tiles that touch a
// boundary use the clipped per-word form above.

// One window for the WPT words of a lane in a warp tile (words
// w0 + lane + 32q): word i0 + 32q and the next one, funnel-shifted.  The
// lane's first index i0 is folded into one pointer so that every load of
// the unrolled loop is that pointer plus a constant offset.
//
// Unguarded tiles load each 32-bit word once: the high word of lane l is
// the low word of lane l + 1, and that of lane 31 is the low word of lane 0
// for q + 1, so one extra load (lane 0, q = WPT) and a shuffle per word
// replace the second load (5 % faster at r = 136279841: fewer load
// instructions queue in the LSU).
template <bool GUARD>
GF2E_DEV void window_at(const u32 *__restrict__ in32, u32 i0, u32 n32, u32 sh,
                        u32 (&acc)[WPT]) {
    const u32 *__restrict__ p = in32 + i0;
    if (!GUARD) {
        const u32 lane = threadIdx.x & 31;
        u32 lo[WPT + 1];
#pragma unroll
        for (int q = 0; q < WPT; q++) lo[q] = __ldg(p + 32 * q);
        lo[WPT] = lane == 0 ? __ldg(p + 32 * WPT) : 0u;
#pragma unroll
        for (int q = 0; q < WPT; q++) {
            const u32 y = lane == 0 ? lo[q + 1] : lo[q];
            const u32 hi = __shfl_sync(0xffffffffu, y, (lane + 1) & 31);
            acc[q] ^= __funnelshift_r(lo[q], hi, sh);
        }
    } else {
#pragma unroll
        for (int q = 0; q < WPT; q++) {
            const u32 lo = (i0 + 32 * q < n32) ? __ldg(p + 32 * q) : 0u;
            const u32 hi = (i0 + 32 * q + 1 < n32) ? __ldg(p + 32 * q + 1) : 0u;
            acc[q] ^= __funnelshift_r(lo, hi, sh);
        }
    }
}
// The window starting at input bit 32 w + K.  The highest index the warp
// reads is w0 + 32 WPT + (K >> 5) (the high word of lane 31 at q = WPT - 1,
// loaded by lane 0 as its word for q = WPT); tiles whose highest index is
// inside the state skip the bounds tests.  Every lane of the warp takes the
// same branch (the test depends on w0 and K only), as the shuffle needs.
GF2E_DEV void window_strided(const u32 *__restrict__ in32, u32 wl, u32 w0, u32 n32, u32 K,
                             u32 (&acc)[WPT]) {
    const u32 off = K >> 5;
    if (w0 + 32 * WPT + off < n32)
        window_at<false>(in32, wl + off, n32, K & 31, acc);
    else
        window_at<true>(in32, wl + off, n32, K & 31, acc);
}

// A clean warp tile of 32*WPT words: lane handles words w0 + lane + 32q, so
// every load and store instruction of the warp touches consecutive words.
template <bool SODD>
GF2E_DEV void square_tile_fast(const u32 *__restrict__ in32, u32 n32, u32 w0, u32 lane,
                               bool t1_on, bool t3_on, bool t4_on, bool t5_on, u32 K2, u32 K3,
                               u32 K4, u32 K5, u64 *__restrict__ o) {
    u32 E[WPT], O[WPT];
    const u32 wl = w0 + lane;
    const u32 *__restrict__ p1 = in32 + wl;
#pragma unroll
    for (int q = 0; q < WPT; q++) {
        E[q] = t1_on ? __ldg(p1 + 32 * q) : 0u;
        O[q] = 0;
    }
    window_strided(in32, wl, w0, n32, K2, O);
    if (t3_on) window_strided(in32, wl, w0, n32, K3, SODD ? E : O);
    if (t4_on) window_strided(in32, wl, w0, n32, K4, SODD ? O : E);
    if (t5_on) window_strided(in32, wl, w0, n32, K5, E);
    u64 *__restrict__ op = o + wl;
#pragma unroll
    for (int q = 0; q < WPT; q++) op[32 * q] = interleave32(E[q], O[q]);
}

// Batched squaring: blockIdx.y = state, warps stride over the state's tiles.
// All clean-tile conditions use 32-bit arithmetic (bit positions < 2^32
// for r < 2^31); larger r take the clipped per-word path throughout.
__global__ void __launch_bounds__(256, 4)
k_square_batch(const u64 *__restrict__ in, u64 *__restrict__ out, size_t stride,
               u64 r, const u64 *__restrict__ s_arr, u64 s_uniform) {
    const int st = blockIdx.y;
    const u64 s = s_arr ? s_arr[st] : s_uniform;
    const u32 nw = (u32)((r + 63) >> 6);
    const u32 n32 = 2 * nw;
    const u64 h = (r + 1) >> 1;
    const u32 *in32 = reinterpret_cast<const u32 *>(in + (size_t)st * stride);
    u64 *o = out + (size_t)st * stride;
    // window geometry: input bit position of word w's window is 32w + K
    const u32 K2 = (u32)h;                                 // S << 1
    const u32 K3 = (u32)(h - ((s + 1) >> 1));              // S << (s+1)
    const u32 K4 = (u32)(h + ((r - s) >> 1));              // S >> (r-s-1)
    const u32 K5 = (u32)(h + ((r - 2 * s) >> 1));          // (S >> (r-s-1)) << s
    const bool sodd = (s & 1) != 0;
    const bool small_r = r < (1ull << 31);
    const u32 s32 = (u32)s, h32 = (u32)h, c3 = (u32)((s + 1) >> 1);
    // warp tiles of TW words; the clean test is the same for the whole warp
    constexpr u32 TW = 32 * WPT;
    const u32 lane = threadIdx.x & 31;
    const u32 ntiles = (nw + TW - 1) / TW;
    const u32 warps_total = (gridDim.x * blockDim.x) >> 5;
    for (u32 t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < ntiles; t += warps_total) {
        const u32 w0 = TW * t;
        bool clean = false, t1_on = false, t3_on = false, t4_on = false, t5_on = false;
        if (small_r && w0 + TW + 1 <= nw) {
            const u32 b0 = w0 << 6, bl = b0 + 64 * (TW - 1);      // first/last word bit
            t1_on = 32 * (w0 + TW) <= h32;
            const bool t1_off = 32 * w0 >= h32;
            t4_on = bl + 1 < s32;
            const bool t4_off = b0 + 1 >= s32;
            t5_on = b0 >= s32 && bl + 1 < 2 * s32;
            const bool t5_off = bl + 64 <= s32 || b0 + 1 >= 2 * s32;
            t3_on = 32 * w0 >= c3;
            const bool t3_off = bl + 64 <= s32 + 1;
            clean = (t1_on || t1_off) && (t3_on || t3_off) && (t4_on || t4_off) &&
                    (t5_on || t5_off);
        }
        if (clean) {
            if (sodd)
                square_tile_fast<true>(in32, n32, w0, lane, t1_on, t3_on, t4_on, t5_on, K2, K3,
                                       K4, K5, o);
            else
                square_tile_fast<false>(in32, n32, w0, lane, t1_on, t3_on, t4_on, t5_on, K2, K3,
                                        K4, K5, o);
        } else {
            for (u32 w = w0 + lane; w < w0 + TW && w < nw; w += 32)
                o[w] = square_word(in32, n32, r, h, s, w);
        }
    }
}

// P_hi bits [k, k+64) where P_hi = P >> r, P of L bits in pw words; bits of
// P below r (k < 0) and at or above L are excluded.  Callers pass k >= -s,
// so the absolute position r + k is never negative.
GF2E_DEV u64 phi_window(const u64 *__restrict__ P, size_t pw, u64 r, u64 L, int64_t k) {
    int64_t q = (int64_t)r + k;                   // absolute bit position
    u64 lo_clip = 0;
    if (k < 0) {
        lo_clip = (u64)(-k);
        if (lo_clip >= 64) return 0;
    }
    u64 pos = (u64)q;
    if (pos >= L) return 0;
    size_t i = (size_t)(pos >> 6);
    unsigned sh = (unsigned)(pos & 63);
    u64 a = (i < pw) ? P[i] : 0;
    u64 b2 = (i + 1 < pw) ? P[i + 1] : 0;
    u64 v = funnel64(a, b2, sh);
    if (L - pos < 64) v &= low_mask(L - pos);
    if (lo_clip) v &= ~low_mask(lo_clip);
    return v;
}

// out = P mod T for a product P of L <= 2r-1 bits (five windows of P_hi).
// Batched: blockIdx.y selects P + y*pstride, out + y*ostride and s_arr[y].
__global__ void k_reduce(const u64 *__restrict__ P, size_t pw, u64 L, u64 *__restrict__ out,
                         u64 r, u64 s, size_t pstride = 0, size_t ostride = 0,
                         const u64 *__restrict__ s_arr = nullptr) {
    P += (size_t)blockIdx.y * pstride;
    out += (size_t)blockIdx.y * ostride;
    if (s_arr) s = s_arr[blockIdx.y];
    const size_t nw = (size_t)((r + 63) >> 6);
    for (size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x; w < nw;
         w += (size_t)gridDim.x * blockDim.x) {
        const u64 b = (u64)w << 6;
        u64 v = (w < pw) ? P[w] : 0;                  // P_lo
        if (b + 64 > r) v &= low_mask(r > b ? r - b : 0);
        if (b >= L) v = 0;
        else if (L - b < 64) v &= low_mask(L - b);
        v ^= phi_window(P, pw, r, L, (int64_t)b);                    // P_hi
        u64 y = phi_window(P, pw, r, L, (int64_t)b - (int64_t)s);    // P_hi<<s
        if (b + 64 > r) y &= low_mask(r - b);
        v ^= y;
        v ^= phi_window(P, pw, r, L, (int64_t)(b + r - s));          // Q
        u64 z = phi_window(P, pw, r, L, (int64_t)(b + r) - 2 * (int64_t)s);  // Q<<s
        if (b < s) z &= (s - b >= 64) ? 0 : ~low_mask(s - b);
        v ^= z;
        out[w] = v;
    }
}

__global__ void k_set_const(u64 *states, size_t stride, int nstates, size_t nw, u64 w0) {
    size_t total = (size_t)nstates * stride;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        size_t w = i % stride;
        states[i] = (w == 0) ? w0 : 0;
        (void)nw;
    }
}

int check_rs(u64 r, u64 s) {
    if (r < 5 || !(r & 1))
        return gf2e::invalid("r must be odd and >= 5 (got %llu)", (unsigned long long)r);
    if (!(s >= 1 && 2 * s < r))
        return gf2e::invalid("need 1 <= s <= (r-1)/2 (r=%llu s=%llu)",
                             (unsigned long long)r, (unsigned long long)s);
    return GF2E_OK;
}

int launch_square(const u64 *in, u64 *out, size_t stride, int nstates, u64 r,
                  const u64 *s_dev, u64 s, cudaStream_t st) {
    const size_t nw = (size_t)((r + 63) >> 6);
    const int threads = 256;
    // Two warp tiles per warp spread the per-state setup over 16 words a
    // thread (one tile per warp measured 8 % slower at r = 136279841), when
    // the grid still fills every SM (4 blocks each) at least four times;
    // small states (r ~ 10^6) keep one tile per warp and twice the blocks.
    const size_t tile_words = (size_t)WPT * threads;
    const size_t wide_blocks = (nw + 2 * tile_words - 1) / (2 * tile_words);
    const bool two = wide_blocks * (size_t)nstates >= (size_t)16 * gf2e::sm_count();
    const size_t per_block = two ? 2 * tile_words : tile_words;
    size_t bx = (nw + per_block - 1) / per_block;
    if (bx > 65535) bx = 65535;
    dim3 grid((unsigned)bx, (unsigned)nstates);
    k_square_batch<<<grid, threads, 0, st>>>(in, out, stride, r, s_dev, s);
    GF2E_CHECK_LAUNCH("k_square_batch");
    return GF2E_OK;
}

}  // namespace

namespace gf2e {
int frobenius_states(u64 *a, u64 *b, size_t stride, int nstates, u64 r, const u64 *s_dev,
                     u64 k, cudaStream_t st, u64 s_uniform = 0);
int trin_reduce(const u64 *P, size_t pw, u64 L, u64 *out, u64 r, u64 s, cudaStream_t st) {
    const size_t nw = (size_t)((r + 63) >> 6);
    int threads = 256;
    k_reduce<<<grid_for(nw, threads), threads, 0, st>>>(P, pw, L, out, r, s);
    GF2E_CHECK_LAUNCH("k_reduce");
    return GF2E_OK;
}
int trin_reduce_batch(const u64 *P, size_t pstride, size_t pw, u64 L, u64 *out, size_t ostride,
                      u64 r, const u64 *s_dev, int batch, cudaStream_t st) {
    const size_t nw = (size_t)((r + 63) >> 6);
    int per = std::max(1, grid_for(nw, 256) / batch);
    k_reduce<<<dim3(per, batch), 256, 0, st>>>(P, pw, L, out, r, 0, pstride, ostride, s_dev);
    GF2E_CHECK_LAUNCH("k_reduce batch");
    return GF2E_OK;
}
int trin_square_states(const u64 *in, u64 *out, size_t stride, int nstates, u64 r,
                       const u64 *s_dev, cudaStream_t st) {
    return launch_square(in, out, stride, nstates, r, s_dev, 0, st);
}
int trin_square_any(const u64 *in, u64 *out, size_t stride, int nstates, u64 r,
                    const u64 *s_dev, u64 s, cudaStream_t st) {
    return launch_square(in, out, stride, nstates, r, s_dev, s, st);
}
int trin_square(const u64 *in, u64 *out, u64 r, u64 s, cudaStream_t st) {
    return launch_square(in, out, (size_t)((r + 63) >> 6), 1, r, nullptr, s, st);
}
int trin_set_const(u64 *states, size_t stride, int nstates, u64 r, u64 w0, cudaStream_t st) {
    const size_t nw = (size_t)((r + 63) >> 6);
    size_t total = (size_t)nstates * stride;
    int threads = 256;
    k_set_const<<<grid_for(total, threads), threads, 0, st>>>(states, stride, nstates, nw, w0);
    GF2E_CHECK_LAUNCH("k_set_const");
    return GF2E_OK;
}
}  // namespace gf2e

extern "C" {

int gf2e_trin_square(const uint64_t *in_dev, uint64_t *out_dev, uint64_t r, uint64_t s,
                     void *stream) {
    GF2E_TRY(check_rs(r, s));
    if (!in_dev || !out_dev || in_dev == out_dev)
        return gf2e::invalid("gf2e_trin_square: need distinct non-null buffers");
    return gf2e::trin_square(in_dev, out_dev, r, s, (cudaStream_t)stream);
}

int gf2e_trin_square_batch(uint64_t *states_dev, uint64_t *scratch_dev, size_t stride_words,
                           int nstates, uint64_t r, const uint64_t *s_dev, uint32_t k,
                           void *stream) {
    GF2E_TRY(check_rs(r, 1));
    const size_t nw = (size_t)((r + 63) >> 6);
    if (!states_dev || !scratch_dev || !s_dev || nstates < 1 || nstates > 65535)
        return gf2e::invalid("gf2e_trin_square_batch: bad buffers or nstates=%d", nstates);
    if (stride_words < nw || (stride_words & 1))
        return gf2e::invalid("stride_words must be even and >= ceil(r/64)");
    return gf2e::frobenius_states(states_dev, scratch_dev, stride_words, nstates, r, s_dev, k,
                                  (cudaStream_t)stream);
}

int gf2e_trin_set_x(uint64_t *states_dev, size_t stride_words, int nstates, uint64_t r,
                    void *stream) {
    if (!states_dev || nstates < 1 || stride_words < (size_t)((r + 63) >> 6) || r < 2)
        return gf2e::invalid("gf2e_trin_set_x: bad arguments");
    return gf2e::trin_set_const(states_dev, stride_words, nstates, r, 2, (cudaStream_t)stream);
}

int gf2e_trin_set_one(uint64_t *states_dev, size_t stride_words, int nstates, uint64_t r,
                      void *stream) {
    if (!states_dev || nstates < 1 || stride_words < (size_t)((r + 63) >> 6) || r < 1)
        return gf2e::invalid("gf2e_trin_set_one: bad arguments");
    return gf2e::trin_set_const(states_dev, stride_words, nstates, r, 1, (cudaStream_t)stream);
}

}  // extern "C"

namespace {

// The host-buffer entry point's device workspace, its copy stream and event:
// one set per host thread, kept between calls, released on a device switch
// (on the device that owns them) and when the thread exits.
struct FrobeniusWorkspace {
    u64 *buf = nullptr;
    size_t bytes = 0;
    int dev = -1;
    cudaStream_t copy_st = nullptr;
    cudaEvent_t ev_done = nullptr;
    int copy_dev = -1;

    template <class F>
    static void on_device(int dev, F &&f) {
        int cur = -1;
        if (cudaGetDevice(&cur) != cudaSuccess) return;
        if (cur != dev && cudaSetDevice(dev) != cudaSuccess) return;
        f();
        if (cur != dev) cudaSetDevice(cur);
    }
    void release_buffer() {
        if (buf) on_device(dev, [&] { cudaFree(buf); });
        buf = nullptr;
        bytes = 0;
        dev = -1;
    }
    void release_stream() {
        if (copy_st || ev_done)
            on_device(copy_dev < 0 ? 0 : copy_dev, [&] {
                if (ev_done) cudaEventDestroy(ev_done);
                if (copy_st) cudaStreamDestroy(copy_st);
            });
        copy_st = nullptr;
        ev_done = nullptr;
        copy_dev = -1;
    }
    ~FrobeniusWorkspace() {
        release_buffer();
        release_stream();
    }
};

FrobeniusWorkspace &frobenius_workspace() {
    static thread_local FrobeniusWorkspace w;
    return w;
}

}  // namespace

extern "C" {

int gf2e_trin_frobenius_host(uint64_t r, const uint64_t *s_host, int nstates, uint32_t k,
                             uint64_t *out_host, size_t out_stride_words, void *stream) {
    GF2E_TRY(check_rs(r, 1));
    const size_t nw = (size_t)((r + 63) >> 6);
    if (!s_host || !out_host || nstates < 1 || nstates > 65535 || out_stride_words < nw)
        return gf2e::invalid("gf2e_trin_frobenius_host: bad arguments");
    for (int i = 0; i < nstates; i++) GF2E_TRY(check_rs(r, s_host[i]));
    cudaStream_t st = (cudaStream_t)stream;
    const size_t stride = nw + (nw & 1);
    const size_t need = 2 * stride * (size_t)nstates * 8 + (size_t)nstates * 8;
    // per-thread device workspace, grown on demand and kept between calls
    FrobeniusWorkspace &W = frobenius_workspace();
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return gf2e::cuda_status(e, "cudaGetDevice");
    if (W.bytes < need || W.dev != dev) {
        W.release_buffer();
        e = cudaMalloc(&W.buf, need);
        if (e != cudaSuccess) {
            W.buf = nullptr;
            return gf2e::cuda_status(e, "frobenius workspace");
        }
        W.bytes = need;
        W.dev = dev;
    }
    u64 *states = W.buf, *scratch = W.buf + stride * nstates, *sdev = scratch + stride * nstates;
    e = cudaMemcpyAsync(sdev, s_host, (size_t)nstates * 8, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return gf2e::cuda_status(e, "frobenius s upload");
    GF2E_TRY(gf2e::trin_set_const(states, stride, nstates, r, 2, st));
    // Large batches go in groups, one after another on `st`, each group's
    // readback on a copy stream while the next group squares, so only the
    // last group's copy adds to the time.  Group sizes shrink towards the
    // end (..., 64, 16, 4 states; the first group takes the rest): a
    // group's readback (17 MB a state at r = 136279841) takes well under
    // the squaring time of a group a quarter its size for any k worth
    // batching, the large first group keeps most launches wide, and the
    // exposed last copy is 4 states.
    const bool split = nstates >= 8 && (size_t)nstates * nw * 8 >= ((size_t)256 << 20);
    if (!split) {
        GF2E_TRY(gf2e_trin_square_batch(states, scratch, stride, nstates, r, sdev, k, stream));
        e = cudaMemcpy2DAsync(out_host, out_stride_words * 8, states, stride * 8, nw * 8,
                              (size_t)nstates, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        return gf2e::cuda_status(e, "frobenius readback");
    }
    int groups[32], ngroups = 0, left = nstates;
    for (int sz = 4; left > sz && ngroups < 31; sz *= 4) {
        groups[ngroups++] = sz;
        left -= sz;
    }
    groups[ngroups++] = left;
    std::reverse(groups, groups + ngroups);
    if (!W.copy_st || W.copy_dev != dev) {
        W.release_stream();
        e = cudaStreamCreateWithFlags(&W.copy_st, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&W.ev_done, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            W.release_stream();
            return gf2e::cuda_status(e, "frobenius copy stream");
        }
        W.copy_dev = dev;
    }
    cudaStream_t copy_st = W.copy_st;
    cudaEvent_t ev_done = W.ev_done;
    for (int gi = 0, g0 = 0; gi < ngroups; g0 += groups[gi], gi++) {
        const int ng = groups[gi];
        GF2E_TRY(gf2e_trin_square_batch(states + stride * g0, scratch + stride * g0, stride, ng,
                                        r, sdev + g0, k, stream));
        e = cudaEventRecord(ev_done, st);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(copy_st, ev_done, 0);
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(out_host + (size_t)g0 * out_stride_words, out_stride_words * 8,
                                  states + stride * g0, stride * 8, nw * 8, (size_t)ng,
                                  cudaMemcpyDeviceToHost, copy_st);
        if (e != cudaSuccess) return gf2e::cuda_status(e, "frobenius group readback");
    }
    e = cudaStreamSynchronize(copy_st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return gf2e::cuda_status(e, "frobenius readback");
}

int gf2e_trin_reduce(const uint64_t *prod_dev, uint64_t prod_bits, uint64_t *out_dev,
                     uint64_t r, uint64_t s, void *stream) {
    GF2E_TRY(check_rs(r, s));
    if (!prod_dev || !out_dev || prod_bits > 2 * r - 1)
        return gf2e::invalid("gf2e_trin_reduce: need prod_bits <= 2r-1");
    size_t pw = (size_t)((prod_bits + 63) >> 6);
    return gf2e::trin_reduce(prod_dev, pw, prod_bits, out_dev, r, s, (cudaStream_t)stream);
}

}  // extern "C"
