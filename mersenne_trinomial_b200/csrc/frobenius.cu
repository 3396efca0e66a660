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
// 4-way bit interleave of C[0..3] (bit 4 t + c = bit t of C[c]): cross-
// register and in-register delta swaps, then a byte transpose by byte
// permutes.  Lanes own units u0 + lane + 32 q, q < 6, so
// loads and 16-byte stores are coalesced.
//
// Per warp tile of 192 units, one ballot lists the windows overlapping it and
// those covering all of it.  The covering windows whose reads stay inside the
// state are applied two at a time (both windows' 32 loads issued before
// either is used) with no masks or bounds tests; the rest (windows that start
// or end inside the tile, a few tiles per state) with per-lane bit masks and
// bounds-tested loads.  The kernel is bound by memory latency and integer
// issue together: measured at r = 136279841, windows one at a time with the
// high words by shuffle ran 1.06 ms a pass (64 states), the per-tile list
// with two loads a unit 0.72 ms, two windows at a time 0.68 ms; staging each
// window's run in shared memory by cp.async first ran 1.5 ms (more issued
// instructions, fewer resident warps).  Each CTA composes its state's
// windows in warp 0 with shifts and masks (the moduli are powers of two).
#include "gf2e_internal.cuh"

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>

namespace {

constexpr int KL = 2;                 // squarings per pass
constexpr int M = 1 << KL;            // residue classes of output bits
constexpr int NCAND = 25;             // 5^KL composed candidates
constexpr u32 UBITS = 32 * M;         // output bits per unit (two words)

struct FWin {
    int lo, hi;       // output bits j in [lo, hi), lo = hi - 1 = c (mod M)
    int K;            // input bit (j - c) / M + K
    int c;
};

struct Win64 {
    int64_t m, c, lo, hi, K;
};

// a mod m in [0, m) for m a power of two (two's complement: the low bits)
GF2E_DEV int64_t mod_pos(int64_t a, int64_t m) { return a & (m - 1); }
GF2E_DEV int log2i(int64_t m) { return 63 - __clzll((unsigned long long)m); }

// window i (0..4) of one squaring; lo >= hi when empty
GF2E_DEV Win64 square_win(int i, int64_t r, int64_t s) {
    const int64_t h = (r + 1) >> 1;
    Win64 w{2, 0, 0, 0, 0};
    switch (i) {
        case 0: w.c = 0; w.lo = 0; w.hi = r; w.K = 0; break;
        case 1: w.c = 1; w.lo = 1; w.hi = r - 1; w.K = h; break;
        case 2: w.c = (s + 1) & 1; w.lo = s + 1; w.hi = r; w.K = h - ((s + 1 - w.c) >> 1); break;
        case 3: w.c = s & 1; w.lo = 0; w.hi = s - 1; w.K = h + ((r - s - 1 + w.c) >> 1); break;
        default: w.c = 0; w.lo = s; w.hi = 2 * s - 1; w.K = h + ((r - 2 * s - 1) >> 1); break;
    }
    return w;
}

// trim [lo, hi) to its first and last member of class c (mod m); the moduli
// are powers of two, so the divisions below are exact shifts
GF2E_DEV void trim(Win64 &w) {
    if (w.lo >= w.hi) return;
    w.lo += mod_pos(w.c - w.lo, w.m);
    if (w.lo < w.hi) w.hi = w.lo + ((w.hi - 1 - w.lo) & ~(w.m - 1)) + 1;
}

// outer window a (modulus 2) applied after inner window b
GF2E_DEV Win64 compose(const Win64 &a, const Win64 &b) {
    Win64 w;
    const int la = log2i(a.m), lb = log2i(b.m);
    w.m = a.m * b.m;
    w.c = a.c + a.m * mod_pos(b.c - a.K, b.m);
    const int64_t t = ((w.c - a.c) >> la) + a.K - b.c;    // a multiple of b.m
    w.K = (t >> lb) + b.K;                                 // exact: arithmetic shift
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

// 4-way bit interleave of one unit: bit 4 t + c of the 128-bit output is
// bit t of C[c].  Index bookkeeping (register index r1 r0, then bit position
// p4..p0): the input holds bit t of class c = (c1 c0) at register (c1 c0),
// position (t4 t3 t2 t1 t0).  Relabelling the registers (free) swaps r1 and
// r0; a cross-register delta swap exchanges r0 with p1, another r1 with p2,
// and one delta swap inside each register exchanges p0 with p2, which gives
// register (t2 t1), position (t4 t3 t0 c1 c0); a 4x4 byte transpose (8 byte
// permutes) then exchanges the register index with the byte index (p4 p3):
// register (t4 t3), position (t2 t1 t0 c1 c0), so register b holds output
// bits [32 b, 32 b + 32).  44 operations for 128 output bits.
GF2E_DEV void xswap(u32 &x, u32 &y, int sh, u32 m) {    // x[p + sh] <-> y[p], p in m
    const u32 t = ((x >> sh) ^ y) & m;
    y ^= t;
    x ^= t << sh;
}
GF2E_DEV u32 dswap(u32 x, int d, u32 m) {                // x[p] <-> x[p + d], p in m
    const u32 t = (x ^ (x >> d)) & m;
    return x ^ (t * (1u + (1u << d)));       // t and t << d are disjoint
}
GF2E_DEV ulonglong2 interleave4(u32 c0, u32 c1, u32 c2, u32 c3) {
    u32 r0 = c0, r1 = c2, r2 = c1, r3 = c3;              // r1 <-> r0 of the index
    xswap(r0, r1, 2, 0x33333333u);                       // r0 <-> p1
    xswap(r2, r3, 2, 0x33333333u);
    xswap(r0, r2, 4, 0x0F0F0F0Fu);                       // r1 <-> p2
    xswap(r1, r3, 4, 0x0F0F0F0Fu);
    r0 = dswap(r0, 3, 0x0A0A0A0Au);                      // p0 <-> p2
    r1 = dswap(r1, 3, 0x0A0A0A0Au);
    r2 = dswap(r2, 3, 0x0A0A0A0Au);
    r3 = dswap(r3, 3, 0x0A0A0A0Au);
    const u32 lo01 = __byte_perm(r0, r1, 0x5140), hi01 = __byte_perm(r0, r1, 0x7362);
    const u32 lo23 = __byte_perm(r2, r3, 0x5140), hi23 = __byte_perm(r2, r3, 0x7362);
    ulonglong2 v;
    v.x = ((u64)__byte_perm(lo01, lo23, 0x7632) << 32) | __byte_perm(lo01, lo23, 0x5410);
    v.y = ((u64)__byte_perm(hi01, hi23, 0x7632) << 32) | __byte_perm(hi01, hi23, 0x5410);
    return v;
}

// ---- the pass: per warp tile, the overlapping windows, two at a time
// units per lane per warp tile (384 words a tile) and resident CTAs per SM:
// measured at r = 136279841 x 64 states, 6 units at 4 CTAs beats 8 at 3 by
// 1.2 % and 4 at 4 by 8 % (a persistent grid of contiguous tile shares was
// 36 % slower than any of them)
constexpr int LANE_UNITS = 6;
constexpr int MIN_CTAS = 4;

// A full window over all of the tile's units, every index inside the state:
// lane l's units u0 + l + 32 q read input words first + l + 32 q and the
// word after it (the high word of the funnel shift) with two plain loads.
template <int UL>
GF2E_DEV void full_window(const u32 *__restrict__ in32, u32 first, u32 lane, u32 sh,
                          u32 (&acc)[UL]) {
    const u32 *__restrict__ p = in32 + (first + lane);
    u32 lo[UL], hi[UL];
#pragma unroll
    for (int q = 0; q < UL; q++) {
        lo[q] = __ldg(p + 32 * q);
        hi[q] = __ldg(p + 32 * q + 1);
    }
#pragma unroll
    for (int q = 0; q < UL; q++) acc[q] ^= __funnelshift_r(lo[q], hi[q], sh);
}

// Two full windows of one class, every load of both issued before use, so
// their memory latencies overlap.
template <int UL>
GF2E_DEV void full_windows2(const u32 *__restrict__ in32, u32 first1, u32 sh1, u32 first2, u32 sh2,
                         u32 lane, u32 (&acc)[UL]) {
    const u32 *__restrict__ p1 = in32 + (first1 + lane);
    const u32 *__restrict__ p2 = in32 + (first2 + lane);
    u32 l1[UL], h1[UL], l2[UL], h2[UL];
#pragma unroll
    for (int q = 0; q < UL; q++) {
        l1[q] = __ldg(p1 + 32 * q);
        h1[q] = __ldg(p1 + 32 * q + 1);
        l2[q] = __ldg(p2 + 32 * q);
        h2[q] = __ldg(p2 + 32 * q + 1);
    }
#pragma unroll
    for (int q = 0; q < UL; q++)
        acc[q] ^= __funnelshift_r(l1[q], h1[q], sh1) ^ __funnelshift_r(l2[q], h2[q], sh2);
}

// Any other overlapping window: per unit the bits t whose output position
// 128 u + c + 4 t lies in [lo, hi), loads bounds-tested.
template <int UL>
GF2E_DEV void part_window(const u32 *__restrict__ in32, u32 n32, u32 u0, u32 lane, FWin w,
                        u32 (&acc)[UL]) {
#pragma unroll
    for (int q = 0; q < UL; q++) {
        const int64_t u = (int64_t)u0 + lane + 32 * q;
        const int64_t j0 = u * UBITS + w.c;
        const int64_t tlo = w.lo > j0 ? (w.lo - j0) / M : 0;
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

// Warp-wide: compose the windows of F -> F^4 mod x^r + x^s + 1 into tab[]
// in class order; returns their number (lane 0's count, on every lane).
GF2E_DEV int compose_windows(u64 r, u64 s, FWin *tab, u32 lane) {
    Win64 w{};
    bool ok = false;
    if (lane < (u32)NCAND) {
        w = candidate((int)lane, (int64_t)r, (int64_t)s);
        ok = w.lo < w.hi;
    }
    int base = 0;
    for (int c = 0; c < M; c++) {
        const u32 b = __ballot_sync(0xffffffffu, ok && w.c == c);
        if (ok && w.c == c) {
            const int pos = base + __popc(b & ((1u << lane) - 1u));
            tab[pos] = FWin{(int)w.lo, (int)w.hi, (int)w.K, c};
        }
        base += __popc(b);
    }
    __syncwarp();
    return base;
}

// One warp tile: the 32 UL units from u0 of one state.  tab[] holds the
// state's nwin windows, `mine` is tab[lane] (lane < nwin).  One ballot lists
// the windows overlapping the tile and another those covering all of it;
// the covering ones whose reads stay inside the state are applied with no
// masks or bounds tests, two of a class at a time.
template <int UL>
GF2E_DEV void frob4_tile(const u32 *__restrict__ in32, ulonglong2 *__restrict__ o, u32 n32,
                         u32 nu, const FWin *tab, int nwin, const FWin &mine, u32 u0, u32 lane) {
    constexpr u32 TWL = 32 * UL;
    const int B0 = (int)(u0 * UBITS), B1 = B0 + (int)(TWL * UBITS);
    const bool over = lane < (u32)nwin && mine.hi > B0 && mine.lo < B1;
    const u32 act = __ballot_sync(0xffffffffu, over);
    const u32 full = __ballot_sync(0xffffffffu, over && mine.lo <= B0 && mine.hi >= B1);
    u32 C[M][UL];
#pragma unroll
    for (int c = 0; c < M; c++)
#pragma unroll
        for (int q = 0; q < UL; q++) C[c][q] = 0;
    for (u32 m = act; m; m &= m - 1) {
        const int k = __ffs(m) - 1;
        const FWin w = tab[k];
        // a full window reads without bounds tests when its highest index,
        // u0 + floor(K/32) + 32 UL (one past the last lane's last word), is
        // inside the state
        const bool fast = ((full >> k) & 1) && (int)u0 + (w.K >> 5) + (int)TWL + 1 < (int)n32;
        if (fast && (m & (m - 1))) {
            const int k2 = __ffs(m & (m - 1)) - 1;
            const FWin w2 = tab[k2];
            const bool fast2 =
                ((full >> k2) & 1) && (int)u0 + (w2.K >> 5) + (int)TWL + 1 < (int)n32;
            if (fast2 && w2.c == w.c) {
                const u32 f1 = (u32)((int)u0 + (w.K >> 5)), f2 = (u32)((int)u0 + (w2.K >> 5));
                const u32 s1 = (u32)w.K & 31u, s2 = (u32)w2.K & 31u;
                switch (w.c) {
                    case 0: full_windows2<UL>(in32, f1, s1, f2, s2, lane, C[0]); break;
                    case 1: full_windows2<UL>(in32, f1, s1, f2, s2, lane, C[1]); break;
                    case 2: full_windows2<UL>(in32, f1, s1, f2, s2, lane, C[2]); break;
                    default: full_windows2<UL>(in32, f1, s1, f2, s2, lane, C[3]); break;
                }
                m &= m - 1;                   // the second window is done too
                continue;
            }
        }
        const u32 first = (u32)((int)u0 + (w.K >> 5)), sh = (u32)w.K & 31u;
        switch (w.c) {            // the class is warp-uniform (one window at a time)
            case 0:
                if (fast) full_window<UL>(in32, first, lane, sh, C[0]);
                else part_window<UL>(in32, n32, u0, lane, w, C[0]);
                break;
            case 1:
                if (fast) full_window<UL>(in32, first, lane, sh, C[1]);
                else part_window<UL>(in32, n32, u0, lane, w, C[1]);
                break;
            case 2:
                if (fast) full_window<UL>(in32, first, lane, sh, C[2]);
                else part_window<UL>(in32, n32, u0, lane, w, C[2]);
                break;
            default:
                if (fast) full_window<UL>(in32, first, lane, sh, C[3]);
                else part_window<UL>(in32, n32, u0, lane, w, C[3]);
                break;
        }
    }
#pragma unroll
    for (int q = 0; q < UL; q++) {
        const u32 u = u0 + lane + 32 * q;
        if (u < nu) o[u] = interleave4(C[0][q], C[1][q], C[2][q], C[3][q]);
    }
}

// Batched F -> F^4 mod T (r < 2^31 - 2^16, even stride): blockIdx.y = state;
// warp 0 composes the state's windows for the CTA, the warps stride over
// its tiles.
__global__ void __launch_bounds__(256, MIN_CTAS)
k_frob4_batch(const u64 *__restrict__ in, u64 *__restrict__ out, size_t stride, u64 r,
              const u64 *__restrict__ s_arr, u64 s_uniform) {
    __shared__ FWin tab[NCAND];
    __shared__ int s_nwin;
    const int st = blockIdx.y;
    const u32 lane = threadIdx.x & 31;
    if (threadIdx.x < 32) {
        const int n = compose_windows(r, s_arr ? s_arr[st] : s_uniform, tab, lane);
        if (lane == 0) s_nwin = n;
    }
    __syncthreads();
    const int nwin = s_nwin;
    const u32 nw = (u32)((r + 63) >> 6);
    const u32 n32 = 2 * nw, nu = (nw + 1) >> 1;
    const u32 *in32 = reinterpret_cast<const u32 *>(in + (size_t)st * stride);
    ulonglong2 *o = reinterpret_cast<ulonglong2 *>(out + (size_t)st * stride);
    const FWin mine = lane < (u32)nwin ? tab[lane] : FWin{0, 0, 0, 0};
    constexpr u32 TWL = 32 * LANE_UNITS;
    const u32 ntiles = (nu + TWL - 1) / TWL;
    const u32 warps_total = (gridDim.x * blockDim.x) >> 5;
    for (u32 t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < ntiles; t += warps_total)
        frob4_tile<LANE_UNITS>(in32, o, n32, nu, tab, nwin, mine, TWL * t, lane);
}

}  // namespace

namespace gf2e {

bool frob4_supported(u64 r, size_t stride) {
    return r < (1ull << 31) - (1ull << 16) && !(stride & 1);
}

// squarings fused per pass for the batched entry points, from
// GF2E_SQUARINGS_PER_PASS (read at each call): 1 keeps the one-squaring
// kernel throughout, 2 uses the fused pass wherever it applies; unset, the
// fused pass is used where it applies and the states do not fit in L2.
int squarings_per_pass() {
    const char *e = getenv("GF2E_SQUARINGS_PER_PASS");
    if (!e) return 0;
    const int v = atoi(e);
    return v == 1 || v == 2 ? v : 0;
}

// fused pass for this batch: applies (r, stride) and pays (not in L2), or forced
bool use_frob4(u64 r, size_t stride, int nstates) {
    const int mode = squarings_per_pass();
    if (mode == 1 || !frob4_supported(r, stride)) return false;
    if (mode == 2) return true;
    // the fused pass halves the HBM traffic per squaring but issues more
    // instructions per byte: when the states and their scratch fit in L2
    // (measured: 256 states at r ~ 10^6, 64 MB, 7 % slower fused) the
    // one-squaring pass is kept
    return (size_t)nstates * stride * 16 > ((size_t)96 << 20);
}


int launch_frob4(const u64 *in, u64 *out, size_t stride, int nstates, u64 r, const u64 *s_dev,
                 u64 s, cudaStream_t st) {
    if (!frob4_supported(r, stride)) return invalid("launch_frob4: needs r < 2^31, even stride");
    const size_t nw = (size_t)((r + 63) >> 6);
    const size_t nu = (nw + 1) / 2;
    // each warp takes four warp tiles (the window set each CTA composes then
    // serves 32 tiles) when that still gives every SM 1.5 rounds of its 4
    // resident CTAs, else one (small states, r ~ 10^6)
    const size_t twl = 32 * (size_t)LANE_UNITS;
    const size_t ntile = (nu + twl - 1) / twl;
    const bool four = (ntile + 31) / 32 * (size_t)nstates >= (size_t)6 * sm_count();
    size_t bx = four ? (ntile + 31) / 32 : (ntile + 7) / 8;
    if (bx > 65535) bx = 65535;
    const dim3 grid((unsigned)bx, (unsigned)nstates);
    k_frob4_batch<<<grid, 256, 0, st>>>(in, out, stride, r, s_dev, s);
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
    const bool fused = use_frob4(r, stride, nstates);
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

extern "C" int gf2e_trin_squarings_per_pass(uint64_t r, size_t stride_words, int nstates) {
    return gf2e::use_frob4(r, stride_words, nstates < 1 ? 1 : nstates) ? 2 : 1;
}
