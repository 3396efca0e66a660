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
// register delta swaps, a byte transpose by byte permutes, then two delta
// swaps inside each 32 bits.
// Lanes own consecutive units (coalesced 16-byte stores).
//
// Memory: a warp tile of 128 units needs, per window overlapping it, one
// contiguous run of 129 input words.  The warp first issues asynchronous
// 16-byte copies (cp.async, zero-filled past the state's ends) of every
// such run into its shared-memory slots, so all of the tile's windows are
// in flight together, then waits once and computes from shared memory.
// (Reading each window straight from global memory serialises one memory
// latency per window: measured 3x slower.)  Windows that cover the whole
// tile are applied unmasked; the few that start or end inside it apply a
// per-lane mask of their output bits.
#include "gf2e_internal.cuh"

#include <algorithm>
#include <atomic>
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

// 4-way bit interleave of one unit: bit 4 t + c of the 128-bit output is
// bit t of C[c].  Index bookkeeping (register index, then bit position): the
// input holds bit t of class c = (c1 c0) at register (c1 c0), position
// (t4 t3 t2 t1 t0).  Two cross-register delta swaps exchange register bit 0
// with position bit 0 and register bit 1 with position bit 1, giving
// register (t1 t0), position (t4 t3 t2 c1 c0); a 4x4 byte transpose (8 byte
// permutes) exchanges the register index with the byte index, giving
// register (t4 t3), position (t1 t0 t2 c1 c0); two delta swaps inside each
// register rotate its position bits to (t2 t1 t0 c1 c0), so register b
// holds output bits [32 b, 32 b + 32).
GF2E_DEV void xswap(u32 &x, u32 &y, int sh, u32 m) {    // x[p + sh] <-> y[p], p in m
    const u32 t = ((x >> sh) ^ y) & m;
    y ^= t;
    x ^= t << sh;
}
GF2E_DEV u32 dswap(u32 x, int d, u32 m) {                // x[p] <-> x[p + d], p in m
    const u32 t = (x ^ (x >> d)) & m;
    return x ^ (t * (1u + (1u << d)));       // t and t << d are disjoint
}
GF2E_DEV u32 rot_pos(u32 x) {                            // (t1 t0 t2 c1 c0) -> (t2 t1 t0 c1 c0)
    return dswap(dswap(x, 4, 0x00F000F0u), 8, 0x0000FF00u);
}
GF2E_DEV ulonglong2 interleave4(u32 c0, u32 c1, u32 c2, u32 c3) {
    xswap(c0, c1, 1, 0x55555555u);
    xswap(c2, c3, 1, 0x55555555u);
    xswap(c0, c2, 2, 0x33333333u);
    xswap(c1, c3, 2, 0x33333333u);
    const u32 lo01 = __byte_perm(c0, c1, 0x5140), hi01 = __byte_perm(c0, c1, 0x7362);
    const u32 lo23 = __byte_perm(c2, c3, 0x5140), hi23 = __byte_perm(c2, c3, 0x7362);
    const u32 o0 = rot_pos(__byte_perm(lo01, lo23, 0x5410));
    const u32 o1 = rot_pos(__byte_perm(lo01, lo23, 0x7632));
    const u32 o2 = rot_pos(__byte_perm(hi01, hi23, 0x5410));
    const u32 o3 = rot_pos(__byte_perm(hi01, hi23, 0x7632));
    ulonglong2 v;
    v.x = ((u64)o1 << 32) | o0;
    v.y = ((u64)o3 << 32) | o2;
    return v;
}

constexpr int WARPS = 8;                           // 256 threads per CTA
constexpr int SLOT_WORDS = TWU + 8;                // a window's run, 16-byte aligned start
constexpr size_t SMEM_BYTES = (size_t)WARPS * NCAND * SLOT_WORDS * sizeof(u32);

// 16-byte asynchronous global -> shared copy of `bytes` (0..16) source
// bytes, the rest of the 16 zero-filled
GF2E_DEV void cp_async16(u32 *dst, const u32 *src, u32 bytes) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(src), "r"(bytes)
                 : "memory");
}

// Stage window w's input run for the tile at unit u0 into `slot`: words
// [base, base + 4 nch) with base = (u0 + floor(K/32)) rounded down to a
// multiple of 4; words outside [0, n32) read as zero.  Word u0 + floor(K/32)
// lands at slot offset (u0 + floor(K/32)) mod 4.
GF2E_DEV void stage_window(const u32 *__restrict__ in32, u32 n32, u32 u0, int K, u32 lane,
                          u32 *slot) {
    const int64_t first = (int64_t)u0 + (K >> 5);
    const int64_t base = first & ~(int64_t)3;
    const int delta = (int)(first - base);
    const int nch = (delta + (int)TWU + 1 + 3) >> 2;
    for (int ch = (int)lane; ch < nch; ch += 32) {
        const int64_t g = base + 4 * ch;
        u32 bytes = 0;
        if (g >= 0 && g < (int64_t)n32) {
            const int64_t left = (int64_t)n32 - g;
            bytes = left >= 4 ? 16u : (u32)(4 * left);
        }
        cp_async16(slot + 4 * ch, bytes ? in32 + g : in32, bytes);
    }
}

// Apply one staged window to the lane's units: input bits 32 u + K + t,
// t = 0..31, are the slot's words i and i + 1 funnel-shifted by K mod 32.
// Windows that start or end inside the tile keep only the bits t whose
// output position 128 u + c + 4 t lies in [lo, hi).
GF2E_DEV void apply_window(const u32 *slot, int delta, u32 u0, u32 lane, FWin w, bool full,
                           u32 (&acc)[UPT]) {
    const u32 sh = (u32)w.K & 31u;
    const u32 *p = slot + delta + lane;
#pragma unroll
    for (int q = 0; q < UPT; q++) {
        u32 v = __funnelshift_r(p[32 * q], p[32 * q + 1], sh);
        if (!full) {
            const int64_t u = (int64_t)u0 + lane + 32 * q;
            const int64_t j0 = u * UBITS + w.c;                  // class bit t = 0
            const int64_t tlo = w.lo > j0 ? (w.lo - j0) / M : 0;
            int64_t thi = w.hi > j0 ? (w.hi - 1 - j0) / M + 1 : 0;
            if (thi > 32) thi = 32;
            u32 mask = 0;
            if (tlo < thi)
                mask = (thi == 32 ? 0xffffffffu : ((1u << thi) - 1u)) & ~((1u << tlo) - 1u);
            v &= mask;
        }
        acc[q] ^= v;
    }
}

// Batched F -> F^4 mod T: blockIdx.y = state, warps stride over its tiles.
// Requires r < 2^31 and an even stride (each unit stores two words; the
// word after an odd nw is padding and receives zero).
__global__ void __launch_bounds__(WARPS * 32, 2)
k_frob4_batch(const u64 *__restrict__ in, u64 *__restrict__ out, size_t stride, u64 r,
              const u64 *__restrict__ s_arr, u64 s_uniform) {
    extern __shared__ u32 stage[];
    __shared__ FWin tab[NCAND];
    __shared__ int s_nwin;
    const int st = blockIdx.y;
    const u64 s = s_arr ? s_arr[st] : s_uniform;
    if (threadIdx.x < 32) {
        // warp 0 composes the candidates and lists the non-empty windows by
        // class (tab[] in class order)
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
            if (ok && w.c == c) {
                const int pos = base + __popc(b & ((1u << lane) - 1u));
                tab[pos] = FWin{(int)w.lo, (int)w.hi, (int)w.K, c};
            }
            base += __popc(b);
        }
        if (lane == 0) s_nwin = base;
    }
    __syncthreads();
    const int nwin = s_nwin;
    const u32 nw = (u32)((r + 63) >> 6);
    const u32 n32 = 2 * nw;
    const u32 nu = (nw + 1) >> 1;
    const u32 *in32 = reinterpret_cast<const u32 *>(in + (size_t)st * stride);
    ulonglong2 *o = reinterpret_cast<ulonglong2 *>(out + (size_t)st * stride);
    const u32 lane = threadIdx.x & 31;
    u32 *slots = stage + (size_t)(threadIdx.x >> 5) * NCAND * SLOT_WORDS;
    // the lane's own window (lane < nwin) for the per-tile overlap test
    const FWin mine = lane < (u32)nwin ? tab[lane] : FWin{0, 0, 0, 0};
    const u32 ntiles = (nu + TWU - 1) / TWU;
    const u32 warps_total = (gridDim.x * blockDim.x) >> 5;
    for (u32 t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < ntiles; t += warps_total) {
        const u32 u0 = TWU * t;
        const int64_t B0 = (int64_t)u0 * UBITS, B1 = B0 + (int64_t)TWU * UBITS;
        const bool over = lane < (u32)nwin && mine.hi > B0 && mine.lo < B1;
        const bool cover = over && mine.lo <= B0 && mine.hi >= B1;
        const u32 act = __ballot_sync(0xffffffffu, over);
        const u32 full = __ballot_sync(0xffffffffu, cover);
        // stage every overlapping window's run, then wait once
        int a = 0;
        for (u32 m = act; m; m &= m - 1, a++)
            stage_window(in32, n32, u0, tab[__ffs(m) - 1].K, lane, slots + a * SLOT_WORDS);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        __syncwarp();
        u32 C[M][UPT];
#pragma unroll
        for (int c = 0; c < M; c++)
#pragma unroll
            for (int q = 0; q < UPT; q++) C[c][q] = 0;
        a = 0;
        for (u32 m = act; m; m &= m - 1, a++) {
            const int k = __ffs(m) - 1;
            const FWin w = tab[k];
            const bool fl = (full >> k) & 1;
            const u32 *sl = slots + a * SLOT_WORDS;
            const int delta = (int)(((int64_t)u0 + (w.K >> 5)) & 3);   // as stage_window
            // the class is warp-uniform (one window at a time)
            switch (w.c) {
                case 0: apply_window(sl, delta, u0, lane, w, fl, C[0]); break;
                case 1: apply_window(sl, delta, u0, lane, w, fl, C[1]); break;
                case 2: apply_window(sl, delta, u0, lane, w, fl, C[2]); break;
                default: apply_window(sl, delta, u0, lane, w, fl, C[3]); break;
            }
        }
        __syncwarp();                     // slots are rewritten by the next tile
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
    // four times over (2 resident blocks each), else one
    const size_t tile_units = (size_t)TWU * (threads / 32);
    const size_t wide = (nu + 2 * tile_units - 1) / (2 * tile_units);
    const bool two = wide * (size_t)nstates >= (size_t)8 * sm_count();
    const size_t per_block = two ? 2 * tile_units : tile_units;
    size_t bx = (nu + per_block - 1) / per_block;
    if (bx > 65535) bx = 65535;
    static std::atomic<bool> attr_done[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_done[dev].load(std::memory_order_acquire)) {
        cudaError_t e = cudaFuncSetAttribute(k_frob4_batch,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)SMEM_BYTES);
        if (e != cudaSuccess) return cuda_status(e, "k_frob4_batch smem attribute");
        attr_done[dev].store(true, std::memory_order_release);
    }
    k_frob4_batch<<<dim3((unsigned)bx, (unsigned)nstates), threads, SMEM_BYTES, st>>>(
        in, out, stride, r, s_dev, s);
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
