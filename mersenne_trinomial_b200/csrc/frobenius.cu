// frobenius.cu -- two squarings per pass over HBM: F -> F^4 mod T,
// T = x^r + x^s + 1 (r odd, 1 <= s, 2s < r), batched over many s.
//
// One squaring F -> F^2 mod T is linear over GF(2), and the derivation in
// trinomial.cu writes it as five windows: output bit j, for j in [lo, hi)
// and j = c (mod 2), is the XOR of input bits (j - c)/2 + K over the windows
// covering j (h = (r+1)/2):
//     spread(A_lo)            c = 0,           [0, r),       K = 0
//     S << 1                  c = 1,           [1, r-1),     K = h
//     S << (s+1) mod x^r      c = (s+1) & 1,   [s+1, r),     K = h - (s+1-c)/2
//     S >> (r-s-1)            c = s & 1,       [0, s-1),     K = h + (r-s-1+c)/2
//     (S >> (r-s-1)) << s     c = 0,           [s, 2s-1),    K = h + (r-2s-1)/2
// Composing two window maps gives windows of the same form with modulus
// M = 4: an outer window (2, ca, [loa, hia), Ka) applied to the output of an
// inner one (mB, cb, [lob, hib), Kb) reads the intermediate bit
// p = (j - ca)/2 + Ka, which lies in the inner window when
// j in [ca + 2 (lob - Ka), ca + 2 (hib - Ka)) and p = cb (mod mB), i.e.
//     j = c := ca + 2 ((cb - Ka) mod mB)   (mod 2 mB),
// and then reads input bit (p - cb)/mB + Kb = (j - c)/(2 mB) + K with
//     K = ((c - ca)/2 + Ka - cb)/mB + Kb.
// So F^4 mod T has at most 25 windows (out bit j = c mod 4 in [lo, hi) takes
// input bit (j - c)/4 + K); at r = 136279841 9 to 13 of them overlap a
// given output tile.  The squaring result is the same bits as two passes of
// the one-squaring kernel (the reference's k_square_fused twice,
// tsfactor.cu:128-186), read and written once instead of twice.
//
// Work unit: a lane's unit is two output words (128 bits).  Its bits of
// class c are j = 128 u + c + 4 t, t = 0..31, whose sources are the 32
// consecutive input bits 32 u + K + t: one funnel-shifted 32-bit read per
// window, XORed into the class accumulator C[c].  The unit's output is the
// 4-way bit interleave of C[0..3] (bit 4 t + c = bit t of C[c]): a byte
// transpose by byte permutes, then four delta swaps inside each 32 bits.
// Lanes own consecutive units (coalesced 16-byte stores); windows that cover
// the whole warp tile read without masks, windows that end inside it
// (a few tiles per state) read with a per-lane bit mask and bounds tests.
#include "gf2e_internal.cuh"

#include <algorithm>
#include <cstdlib>

namespace {

constexpr int KL = 2;                 // squarings per pass
constexpr int M = 1 << KL;            // residue classes of output bits
constexpr int NCAND = 25;             // 5^KL composed candidates
constexpr int UPT = 4;                // units (2 words each) per lane per tile
constexpr u32 UBITS = 32 * M;         // output bits per unit
constexpr u32 TWU = 32 * UPT;         // units per warp tile

struct FWin {
    int lo, hi;       // output bits j in [lo, hi), lo = hi - 1 = c (mod M)
    int K;            // input bit (j - c) / M + K
    int c;
};

struct Win64 {
    int64_t m, c, lo, hi, K;
};

GF2E_DEV int64_t mod_pos(int64_t a, int64_t m) {
    int64_t v = a % m;
    return v < 0 ? v + m : v;
}

// window i (0..4) of one squaring; lo >= hi when empty
GF2E_DEV Win64 square_win(int i, int64_t r, int64_t s) {
    const int64_t h = (r + 1) >> 1;
    Win64 w{2, 0, 0, 0, 0};
    switch (i) {
        case 0: w.c = 0; w.lo = 0; w.hi = r; w.K = 0; break;
        case 1: w.c = 1; w.lo = 1; w.hi = r - 1; w.K = h; break;
        case 2: w.c = (s + 1) & 1; w.lo = s + 1; w.hi = r; w.K = h - (s + 1 - w.c) / 2; break;
        case 3: w.c = s & 1; w.lo = 0; w.hi = s - 1; w.K = h + (r - s - 1 + w.c) / 2; break;
        default: w.c = 0; w.lo = s; w.hi = 2 * s - 1; w.K = h + (r - 2 * s - 1) / 2; break;
    }
    return w;
}

// trim [lo, hi) to its first and last member of class c (mod m)
GF2E_DEV void trim(Win64 &w) {
    if (w.lo >= w.hi) return;
    w.lo += mod_pos(w.c - w.lo, w.m);
    if (w.lo < w.hi) w.hi = w.lo + w.m * ((w.hi - 1 - w.lo) / w.m) + 1;
}

// outer window a (modulus 2) applied after inner window b
GF2E_DEV Win64 compose(const Win64 &a, const Win64 &b) {
    Win64 w;
    w.m = a.m * b.m;
    w.c = a.c + a.m * mod_pos(b.c - a.K, b.m);
    const int64_t t = (w.c - a.c) / a.m + a.K - b.c;      // divisible by b.m
    w.K = t / b.m + b.K;
    w.lo = max(a.lo, a.c + a.m * (b.lo - a.K));
    w.hi = min(a.hi, a.c + a.m * (b.hi - a.K));
    trim(w);
    return w;
}

// candidate i = (outer digit i / 5, inner digit i % 5) for KL = 2
GF2E_DEV Win64 candidate(int i, int64_t r, int64_t s) {
    Win64 in = square_win(i % 5, r, s);
    if (in.lo >= in.hi) return in;
    trim(in);
    if (in.lo >= in.hi) return in;
    Win64 out = square_win(i / 5, r, s);
    if (out.lo >= out.hi) return out;
    return compose(out, in);
}

// 4-way bit interleave of one unit: returns the two output words
GF2E_DEV u32 dswap(u32 x, int d, u32 m) {
    u32 t = (x ^ (x >> d)) & m;
    return x ^ (t * (1u + (1u << d)));       // t and t << d are disjoint
}
GF2E_DEV u32 rot_idx(u32 x) {                // bit 8c + t' -> bit 4t' + c
    x = dswap(x, 7, 0x00AA00AAu);
    x = dswap(x, 14, 0x0000CCCCu);
    x = dswap(x, 4, 0x00F000F0u);
    return dswap(x, 8, 0x0000FF00u);
}
GF2E_DEV ulonglong2 interleave4(u32 c0, u32 c1, u32 c2, u32 c3) {
    const u32 lo01 = __byte_perm(c0, c1, 0x5140), hi01 = __byte_perm(c0, c1, 0x7362);
    const u32 lo23 = __byte_perm(c2, c3, 0x5140), hi23 = __byte_perm(c2, c3, 0x7362);
    const u32 o0 = rot_idx(__byte_perm(lo01, lo23, 0x5410));
    const u32 o1 = rot_idx(__byte_perm(lo01, lo23, 0x7632));
    const u32 o2 = rot_idx(__byte_perm(hi01, hi23, 0x5410));
    const u32 o3 = rot_idx(__byte_perm(hi01, hi23, 0x7632));
    ulonglong2 v;
    v.x = ((u64)o1 << 32) | o0;
    v.y = ((u64)o3 << 32) | o2;
    return v;
}

// A window covering every unit of the tile: lane l's units are
// u0 + l + 32 q, each reading input bits [32 u + K, 32 u + K + 32).  As in
// the one-squaring kernel, each 32-bit word is loaded once when the tile's
// highest index is inside the state: the high word of lane l is the low
// word of lane l + 1 (of lane 0 at q + 1 for lane 31), by shuffle.
GF2E_DEV void win_full(const u32 *__restrict__ in32, u32 n32, u32 u0, u32 lane, int K,
                       u32 (&acc)[UPT]) {
    const int off = K >> 5;                  // floor(K / 32)
    const u32 sh = (u32)K & 31u;
    const u32 i0 = u0 + lane + off;          // >= 0: the window covers unit u0's sources
    const u32 *__restrict__ p = in32 + i0;
    if ((int64_t)u0 + 32 * UPT + off < (int64_t)n32) {
        u32 lo[UPT + 1];
#pragma unroll
        for (int q = 0; q < UPT; q++) lo[q] = __ldg(p + 32 * q);
        lo[UPT] = lane == 0 ? __ldg(p + 32 * UPT) : 0u;
#pragma unroll
        for (int q = 0; q < UPT; q++) {
            const u32 y = lane == 0 ? lo[q + 1] : lo[q];
            const u32 hi = __shfl_sync(0xffffffffu, y, (lane + 1) & 31);
            acc[q] ^= __funnelshift_r(lo[q], hi, sh);
        }
    } else {
#pragma unroll
        for (int q = 0; q < UPT; q++) {
            const u32 i = i0 + 32 * q;
            const u32 lo = i < n32 ? __ldg(p + 32 * q) : 0u;
            const u32 hi = i + 1 < n32 ? __ldg(p + 32 * q + 1) : 0u;
            acc[q] ^= __funnelshift_r(lo, hi, sh);
        }
    }
}

// A window that starts or ends inside the tile: per unit, the bits t whose
// output position 128 u + c + 4 t lies in [lo, hi), loads bounds-tested.
GF2E_DEV void win_part(const u32 *__restrict__ in32, u32 n32, u32 u0, u32 lane, FWin w,
                       u32 (&acc)[UPT]) {
#pragma unroll
    for (int q = 0; q < UPT; q++) {
        const int64_t u = (int64_t)u0 + lane + 32 * q;
        const int64_t j0 = u * UBITS + w.c;                  // class bit t = 0
        int64_t tlo = w.lo > j0 ? (w.lo - j0) / M : 0;
        int64_t thi = w.hi > j0 ? (w.hi - 1 - j0) / M + 1 : 0;
        if (thi > 32) thi = 32;
        if (tlo >= thi) continue;
        const u32 mask = (thi == 32 ? 0xffffffffu : ((1u << thi) - 1u)) & ~((1u << tlo) - 1u);
        const int64_t P = 32 * u + w.K;
        const int64_t i = P >> 5;
        const u32 lo = (i >= 0 && i < (int64_t)n32) ? __ldg(in32 + i) : 0u;
        const u32 hi = (i + 1 >= 0 && i + 1 < (int64_t)n32) ? __ldg(in32 + i + 1) : 0u;
        acc[q] ^= __funnelshift_r(lo, hi, (u32)P & 31u) & mask;
    }
}

// Batched F -> F^4 mod T: blockIdx.y = state, warps stride over its tiles.
// Requires r < 2^31 and an even stride (each unit stores two words; the
// word after an odd nw is padding and receives zero).
__global__ void __launch_bounds__(256, 4)
k_frob4_batch(const u64 *__restrict__ in, u64 *__restrict__ out, size_t stride, u64 r,
              const u64 *__restrict__ s_arr, u64 s_uniform) {
    __shared__ FWin tab[NCAND];
    __shared__ int beg[M + 1];
    const int st = blockIdx.y;
    const u64 s = s_arr ? s_arr[st] : s_uniform;
    if (threadIdx.x < 32) {
        // warp 0 composes the candidates and lists the non-empty windows by class
        const int lane = threadIdx.x;
        Win64 w{};
        bool ok = false;
        if (lane < NCAND) {
            w = candidate(lane, (int64_t)r, (int64_t)s);
            ok = w.lo < w.hi;
        }
        int base = 0;
        for (int c = 0; c < M; c++) {
            const u32 b = __ballot_sync(0xffffffffu, ok && w.c == c);
            if (lane == 0) beg[c] = base;
            if (ok && w.c == c) {
                const int pos = base + __popc(b & ((1u << lane) - 1u));
                tab[pos] = FWin{(int)w.lo, (int)w.hi, (int)w.K, c};
            }
            base += __popc(b);
        }
        if (lane == 0) beg[M] = base;
    }
    __syncthreads();
    const u32 nw = (u32)((r + 63) >> 6);
    const u32 n32 = 2 * nw;
    const u32 nu = (nw + 1) >> 1;
    const u32 *in32 = reinterpret_cast<const u32 *>(in + (size_t)st * stride);
    ulonglong2 *o = reinterpret_cast<ulonglong2 *>(out + (size_t)st * stride);
    const u32 lane = threadIdx.x & 31;
    const u32 ntiles = (nu + TWU - 1) / TWU;
    const u32 warps_total = (gridDim.x * blockDim.x) >> 5;
    for (u32 t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < ntiles; t += warps_total) {
        const u32 u0 = TWU * t;
        const int64_t B0 = (int64_t)u0 * UBITS, B1 = B0 + (int64_t)TWU * UBITS;
        u32 C[M][UPT];
#pragma unroll
        for (int c = 0; c < M; c++)
#pragma unroll
            for (int q = 0; q < UPT; q++) C[c][q] = 0;
#pragma unroll
        for (int c = 0; c < M; c++) {
            for (int k = beg[c]; k < beg[c + 1]; k++) {
                const FWin w = tab[k];
                if (w.hi <= B0 || w.lo >= B1) continue;
                if (w.lo <= B0 && w.hi >= B1)
                    win_full(in32, n32, u0, lane, w.K, C[c]);
                else
                    win_part(in32, n32, u0, lane, w, C[c]);
            }
        }
#pragma unroll
        for (int q = 0; q < UPT; q++) {
            const u32 u = u0 + lane + 32 * q;
            if (u < nu) o[u] = interleave4(C[0][q], C[1][q], C[2][q], C[3][q]);
        }
    }
}

}  // namespace

namespace gf2e {

// squarings fused per pass for the batched entry points: 2 (default) or 1
// (GF2E_SQUARINGS_PER_PASS=1 keeps the one-squaring kernel throughout)
int squarings_per_pass() {
    static const int v = [] {
        const char *e = getenv("GF2E_SQUARINGS_PER_PASS");
        return (e && atoi(e) == 1) ? 1 : 2;
    }();
    return v;
}

bool frob4_supported(u64 r, size_t stride) { return r < (1ull << 31) && !(stride & 1); }

int launch_frob4(const u64 *in, u64 *out, size_t stride, int nstates, u64 r, const u64 *s_dev,
                 u64 s, cudaStream_t st) {
    if (!frob4_supported(r, stride)) return invalid("launch_frob4: needs r < 2^31, even stride");
    const size_t nw = (size_t)((r + 63) >> 6);
    const size_t nu = (nw + 1) / 2;
    const int threads = 256;
    // two warp tiles per warp when the grid still fills every SM at least
    // four times over (4 resident blocks each), else one
    const size_t tile_units = (size_t)TWU * (threads / 32);
    const size_t wide = (nu + 2 * tile_units - 1) / (2 * tile_units);
    const bool two = wide * (size_t)nstates >= (size_t)16 * sm_count();
    const size_t per_block = two ? 2 * tile_units : tile_units;
    size_t bx = (nu + per_block - 1) / per_block;
    if (bx > 65535) bx = 65535;
    k_frob4_batch<<<dim3((unsigned)bx, (unsigned)nstates), threads, 0, st>>>(in, out, stride, r,
                                                                          s_dev, s);
    GF2E_CHECK_LAUNCH("k_frob4_batch");
    return GF2E_OK;
}

int trin_square_any(const u64 *in, u64 *out, size_t stride, int nstates, u64 r,
                    const u64 *s_dev, u64 s, cudaStream_t st);

// k squarings of every state (s_dev[i] for state i, s_uniform for all when
// s_dev is null), alternating between a
// and b, the result left in a.  Squarings go two per pass where the fused
// kernel applies; the passes are made even in number (one fused pass turned
// into two single ones when needed), so no copy is needed unless k = 1 or
// only single passes apply and k is odd.
int frobenius_states(u64 *a, u64 *b, size_t stride, int nstates, u64 r, const u64 *s_dev,
                     u64 k, cudaStream_t st, u64 s_uniform) {
    const bool fused = squarings_per_pass() == 2 && frob4_supported(r, stride);
    u64 n4 = fused ? k / 2 : 0, n1 = k - 2 * n4;
    if (((n4 + n1) & 1) && n4 > 0) {
        n4--;
        n1 += 2;
    }
    u64 *x = a, *y = b;
    for (u64 i = 0; i < n4; i++) {
        GF2E_TRY(launch_frob4(x, y, stride, nstates, r, s_dev, s_uniform, st));
        std::swap(x, y);
    }
    for (u64 i = 0; i < n1; i++) {
        GF2E_TRY(trin_square_any(x, y, stride, nstates, r, s_dev, s_uniform, st));
        std::swap(x, y);
    }
    if (x != a) {
        cudaError_t e = cudaMemcpyAsync(a, x, (size_t)nstates * stride * 8,
                                        cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return cuda_status(e, "frobenius copy-back");
    }
    return GF2E_OK;
}

}  // namespace gf2e

extern "C" int gf2e_trin_squarings_per_pass(uint64_t r, size_t stride_words) {
    return (gf2e::squarings_per_pass() == 2 && gf2e::frob4_supported(r, stride_words)) ? 2 : 1;
}
