// hgcd.cu -- subquadratic GF(2)[x] gcd (half-gcd) for r-bit operands.
//
// The reference computes the interval gcd gcd(ACC, T) at r = 136279841 with
// NTL's GF2X GCD (gf2_gcd_ntl.cpp:32-42; a half-gcd over gf2x products,
// ~62 s per gcd on 6 CPU cores) or its hybrid HGCD with GPU multiplies
// (gf2_gcd_ntl.cpp:360-452, GpuMulHook gf2_gcd.h:155-190).  The quadratic
// GPU gcd (gcd.cu) is fine to ~10^6 bits; this file is the r-bit path.
//
// Algorithm (the classical polynomial half-gcd; every matrix is unimodular
// over GF(2), so the gcd is preserved whatever the degrees do, and the
// degree bookkeeping only decides the amount of work):
//
//   hgcd(a, b), deg a = n > deg b, m = ceil(n/2)
//     returns M with (a', b') = M (a, b), deg a' >= m > deg b'
//     if deg b < m: I
//     if n <= H0:   one-CTA Lehmer kernel (64-bit windows, stop at deg b < m)
//     M1 = hgcd(a quo x^m, b quo x^m);  (c, d) = M1 (a, b)
//     if deg d < m: M1
//     one division step c = q d + e; M1 <- [[0,1],[1,q]] M1; (c, d) <- (d, e)
//     if deg d < m: M1
//     k = 2m - deg c;  M2 = hgcd(c quo x^k, d quo x^k);  M2 M1
//
//   gcd(a, b): while deg b >= G0: M = hgcd(a, b); (a, b) = M (a, b); one
//   division step.  Then the quadratic Lehmer gcd (gcd.cu) finishes.
//
// B200 mapping.  The recursion is host-driven on one stream; degrees are
// read back with one small probe per node.  Products are sums of two
// products (matrix x vector and matrix x matrix): a schoolbook carry-less
// kernel split over output words and input chunks (atomicXor partials) below
// a size threshold, the Cantor FFT above it (transforms of a and b shared by
// both rows).  Temporaries come from a per-gcd arena over a private
// stream-ordered memory pool.  A single gcd is latency-bound (the quotient
// sequence is sequential, and its base cases run on one SM each), so
// independent gcds run as a lockstep batch (class HgcdBatch): one host
// thread steps up to 64 of them through the recursion together, every
// launch serving all members with their own sizes (the base cases as one
// grid of a CTA per member, the transforms as batched FFTs); two such
// batches run at once on two streams, one's base cases overlapping the
// other's products.  Run one host thread per gcd instead, 16 gcds of 136
// Mbit kept 16 host cores busy on stream waits and launches while the GPU
// idled between kernels.
#include "gf2e_internal.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <exception>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace gf2e {
int mul_fft_m(u64 abits, u64 bbits);
gf2e_fft_plan *cached_plan(int m);
int fft_fwd_packed(const gf2e_fft_plan *plan, u64 *f, const u32 *src32, u64 nchunks,
                   cudaStream_t st);
int fft_run(const gf2e_fft_plan *plan, bool forward, u64 *f, cudaStream_t st);
int overlap_add(const u64 *F, u64 nchunks, u64 *out, u64 ow, cudaStream_t st);
int fft_fwd_packed_batch(const gf2e_fft_plan *plan, u64 *f, u64 fstride, const u32 *src32,
                         u64 sstride32, u64 nchunks, u64 xor0, int batch, cudaStream_t st);
int fft_run_batch(const gf2e_fft_plan *plan, bool forward, u64 *f, u64 fstride, int batch,
                  cudaStream_t st);
int overlap_add_batch(const u64 *F, u64 fstride, u64 nchunks, u64 *out, u64 ostride, u64 ow,
                      int batch, cudaStream_t st);
u64 fft_plan_n(const gf2e_fft_plan *plan);
}  // namespace gf2e

namespace {

constexpr int BASE_THREADS = 512;
constexpr int GMAX = 64;        // members of one lockstep batch

// ------------------------------------------------------------------ device
GF2E_DEV void clmul64(u64 a, u64 b, u64 &lo, u64 &hi) {
    const u32 a0 = (u32)a, a1 = (u32)(a >> 32), b0 = (u32)b, b1 = (u32)(b >> 32);
    const u64 L = clmul32(a0, b0), H = clmul32(a1, b1);
    const u64 Mid = clmul32(a0 ^ a1, b0 ^ b1) ^ L ^ H;
    lo = L ^ (Mid << 32);
    hi = H ^ (Mid >> 32);
}

GF2E_DEV int deg64(u64 v) { return v ? 63 - __clzll(v) : -1; }

// out = X1*Y1 ^ X2*Y2 pointwise in GF(2^64)
__global__ void k_pw_muladd(u64 *out, const u64 *x1,
                            const u64 *__restrict__ y1, const u64 *__restrict__ x2,
                            const u64 *__restrict__ y2, u64 n) {
    for (u64 k = (u64)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (u64)gridDim.x * blockDim.x) {
        u64 v = gf64_mul(x1[k], y1[k]);
        if (x2) v ^= gf64_mul(x2[k], y2[k]);
        out[k] = v;
    }
}

// ---- lockstep batch: member g of a batched polynomial lives at
// base + g * stride (words); every kernel writes whole member slices, so
// the words above a member's degree are always zero ----

// degree and top window of up to four batched polynomials; block g =
// member, warp w = polynomial (nw = 0: not probed, reads -1)
struct ProbeBatch {
    const u64 *p[4];
    u64 stride[4];
    u32 nw[4][GMAX];
};
__global__ void k_probe_b(const ProbeBatch P, int np, long long *out) {
    const int g = blockIdx.x, w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (w >= np) return;
    const u64 *X = P.p[w] + (u64)g * P.stride[w];
    long long top = -1;
    for (long long base = (long long)P.nw[w][g] - 1; base >= 0 && top < 0; base -= 32) {
        const long long i = base - lane;
        const u64 v = (i >= 0) ? X[i] : 0;
        const unsigned ball = __ballot_sync(0xffffffffu, v != 0);
        if (ball) top = base - (__ffs(ball) - 1);
    }
    if (lane == 0) {
        long long deg = -1;
        u64 win = 0;
        if (top >= 0) {
            const u64 hiw = X[top];
            const int t = 63 - __clzll(hiw);
            deg = top * 64 + t;
            win = hiw << (63 - t);
            if (t < 63 && top > 0) win |= X[top - 1] >> (t + 1);
        }
        out[(g * 4 + w) * 2] = deg;
        out[(g * 4 + w) * 2 + 1] = (long long)win;
    }
}

// member slices dst = src quo x^k[g] (nd[g] words, zero above); blockIdx.y = g
struct ShrBatch {
    const u64 *src;
    u64 *dst;
    u64 ss, ds;
    u64 k[GMAX];
    u32 ns[GMAX], nd[GMAX];
};
__global__ void k_shr_b(const ShrBatch B) {
    const int g = blockIdx.y;
    const u64 *__restrict__ src = B.src + (u64)g * B.ss;
    u64 *__restrict__ dst = B.dst + (u64)g * B.ds;
    const u64 ks = B.k[g] >> 6, ns = B.ns[g], nd = B.nd[g];
    const unsigned kb = (unsigned)(B.k[g] & 63);
    for (u64 w = (u64)blockIdx.x * blockDim.x + threadIdx.x; w < B.ds;
         w += (u64)gridDim.x * blockDim.x) {
        u64 v = 0;
        if (w < nd) {
            const u64 lo = (w + ks < ns) ? src[w + ks] : 0, hi = (w + ks + 1 < ns) ? src[w + ks + 1] : 0;
            v = funnel64(lo, hi, kb);
        }
        dst[w] = v;
    }
}

// up to four sums x1*y1 + x2*y2 per member (schoolbook): thread = two
// adjacent output words, blockIdx.y = a chunk of the x index (partial sums
// XORed into the output, zero on entry), blockIdx.z = job * G + member
struct Mul2Batch {
    const u64 *x1[4], *y1[4], *x2[4], *y2[4];
    u64 sx1[4], sy1[4], sx2[4], sy2[4];
    unsigned long long *out[4];
    u64 so[4];
    u32 nx1[4][GMAX], ny1[4][GMAX], nx2[4][GMAX], ny2[4][GMAX], nout[4][GMAX];
};
__global__ void k_mul2_b(const Mul2Batch J, int G, u64 chunk) {
    const int z = blockIdx.z / G, g = blockIdx.z % G;
    const u64 nout = J.nout[z][g];
    const u64 w = 2 * ((u64)blockIdx.x * blockDim.x + threadIdx.x);
    if (w >= nout) return;
    unsigned long long *__restrict__ out = J.out[z] + (u64)g * J.so[z];
    const u64 i0 = (u64)blockIdx.y * chunk;
    u64 r0 = 0, r1 = 0;
    for (int pr = 0; pr < 2; pr++) {
        const u64 *x = pr ? J.x2[z] : J.x1[z], *y = pr ? J.y2[z] : J.y1[z];
        const u64 nx = pr ? J.nx2[z][g] : J.nx1[z][g], ny = pr ? J.ny2[z][g] : J.ny1[z][g];
        if (!x || !nx || !ny) continue;
        x += (u64)g * (pr ? J.sx2[z] : J.sx1[z]);
        y += (u64)g * (pr ? J.sy2[z] : J.sy1[z]);
        const u64 i1 = min(nx, i0 + chunk);
        for (u64 i = i0; i < i1; i++) {
            const u64 xi = x[i];
            if (!xi) continue;
            u64 lo, hi;
            if (w >= i + 1 && w - 1 - i < ny) { clmul64(xi, y[w - 1 - i], lo, hi); r0 ^= hi; }
            if (w >= i && w - i < ny) { clmul64(xi, y[w - i], lo, hi); r0 ^= lo; r1 ^= hi; }
            if (w + 1 >= i && w + 1 - i < ny) { clmul64(xi, y[w + 1 - i], lo, hi); r1 ^= lo; }
        }
    }
    if (r0) atomicXor(out + w, (unsigned long long)r0);
    if (r1 && w + 1 < nout) atomicXor(out + w + 1, (unsigned long long)r1);
}

// member slices out = x ^ ((q[g] y) << s[g]) below nout[g], zero above
// (q = 0 copies x; out may be x)
struct AxpyBatch {
    u64 *out;
    const u64 *x, *y;
    u64 so, sx, sy;
    u64 q[GMAX], s[GMAX];
    u32 nx[GMAX], ny[GMAX], nout[GMAX];
};
__global__ void k_axpy_b(const AxpyBatch B) {
    const int g = blockIdx.y;
    u64 *out = B.out + (u64)g * B.so;
    const u64 *x = B.x + (u64)g * B.sx;
    const u64 *__restrict__ y = B.y + (u64)g * B.sy;
    const u64 q = B.q[g], nx = B.nx[g], ny = B.ny[g], nout = B.nout[g];
    const u64 sw = B.s[g] >> 6;
    const unsigned sb = (unsigned)(B.s[g] & 63);
    for (u64 w = (u64)blockIdx.x * blockDim.x + threadIdx.x; w < B.so;
         w += (u64)gridDim.x * blockDim.x) {
        u64 v = 0;
        if (w < nout) {
            auto Pw = [&](long long j) -> u64 {         // word j of q * y
                if (!q || j < 0 || j > (long long)ny) return 0;
                u64 r = 0, lo, hi;
                if (j < (long long)ny) { clmul64(q, y[j], lo, hi); r ^= lo; }
                if (j >= 1) { clmul64(q, y[j - 1], lo, hi); r ^= hi; }
                return r;
            };
            const long long j = (long long)w - (long long)sw;
            const u64 shv = sb ? ((Pw(j) << sb) | (Pw(j - 1) >> (64 - sb))) : Pw(j);
            v = (w < nx ? x[w] : 0) ^ shv;
        }
        out[w] = v;
    }
}

// member slices out = (bit g of mask) ? t : f, n words of the chosen, zero above
struct SelectBatch {
    const u64 *t, *f;
    u64 *out;
    u64 st, sf, so;
    unsigned long long mask;
    u32 nt[GMAX], nf[GMAX];
};
__global__ void k_select_b(const SelectBatch B) {
    const int g = blockIdx.y;
    const bool pick = (B.mask >> g) & 1;
    const u64 *__restrict__ src = pick ? B.t + (u64)g * B.st : B.f + (u64)g * B.sf;
    const u64 n = pick ? B.nt[g] : B.nf[g];
    u64 *__restrict__ out = B.out + (u64)g * B.so;
    for (u64 w = (u64)blockIdx.x * blockDim.x + threadIdx.x; w < B.so;
         w += (u64)gridDim.x * blockDim.x)
        out[w] = w < n ? src[w] : 0;
}

// word 0 of every member slice <- 1 (slices zeroed before)
__global__ void k_set_one_b(u64 *p, u64 stride, int G) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < G) p[(u64)g * stride] = 1;
}

// ---- base case: Lehmer half-gcd in one CTA, operands in shared memory ----

GF2E_DEV u64 win_at(const u64 *X, long long nw, long long pos) {   // bits pos..pos+63
    long long i = pos >> 6;
    unsigned sh = (unsigned)(pos & 63);
    u64 a = (i >= 0 && i < nw) ? X[i] : 0, b = (i + 1 < nw) ? X[i + 1] : 0;
    return funnel64(a, b, sh);
}

// totals over the base cases of one gcd, read once when the gcd is done
struct BaseAcc {
    unsigned long long rounds;
    unsigned long long cyc_serial, cyc_total;   // SM clock cycles: thread-0 window phase, total
    int worst;                                  // first non-OK status, else GF2E_OK
};

// warp-wide degree of X below word `top` (inclusive); all 32 lanes return it
GF2E_DEV long long warp_degree(const u64 *X, long long top) {
    const int lane = threadIdx.x & 31;
    for (long long base = top; base >= 0; base -= 32) {
        long long i = base - lane;
        u64 v = (i >= 0) ? X[i] : 0;
        unsigned ball = __ballot_sync(0xffffffffu, v != 0);
        if (ball) {
            int l = __ffs(ball) - 1;
            u64 vv = __shfl_sync(0xffffffffu, v, l);
            return (base - l) * 64 + 63 - __clzll(vv);
        }
    }
    return -1;
}

// one Lehmer round on exact 64-bit windows of A and B taken at bit `lo`
// (deg A = da >= deg B): whole quotients while every bit they depend on is
// exact (a row's window bits are exact above its matrix degree), the
// half-gcd stop (deg B < m) is not reached and the 2x2 matrix stays within
// degree 31; mode 1 (no quotient fits) is the single shift-XOR A ^= B << k.
struct Lehmer {
    u32 mt[4];
    long long k;
    int mode;
};
GF2E_DEV Lehmer lehmer_round(u64 wa, u64 wb, long long da, long long db, long long lo,
                             long long m) {
    Lehmer L;
    u32 ma0 = 1, ma1 = 0, mb0 = 0, mb1 = 1;
    int dga = (int)(da - lo), dgb = deg64(wb), dma = 0, dmb = 0, steps = 0;
    const bool exact = (lo == 0);
    const int dstop = (int)max(-1LL, m - lo);          // window degree of x^m
    // the windows left-aligned (leading coefficient at bit 63): the division
    // below then tests one bit and shifts, with no degree search per step
    u64 A = wa << (63 - dga);
    u64 B = dgb >= 0 ? wb << (63 - dgb) : 0;
    for (int it = 0; it < 64; it++) {
        if (dgb < 0 || dgb < dstop) break;              // b = 0 / half-gcd stop
        const int dq = dga - dgb;
        const int ndm = max(dma, dmb + dq);
        if (ndm > 31) break;                            // matrix degree bound
        if (!exact && dgb < ndm) break;                 // quotient not exact
        // a <- a mod b, row a += q row b: at each of the dq + 1 degrees from
        // the top, XOR in b (and x^(dq-j) row b) when a's leading bit is set,
        // then move one degree down.  Afterwards bit 63 of A is degree dgb.
        // At the top degree the bit is a's leading coefficient, always set.
        u32 s0 = mb0 << dq, s1 = mb1 << dq;
        A ^= B;
        ma0 ^= s0;
        ma1 ^= s1;
#pragma unroll 1
        for (int j = 1; j <= dq; j++) {
            A <<= 1;
            s0 >>= 1;
            s1 >>= 1;
            const u64 msk = (u64)((long long)A >> 63);
            A ^= B & msk;
            ma0 ^= s0 & (u32)msk;
            ma1 ^= s1 & (u32)msk;
        }
        const int c = A ? __clzll(A) : 64;
        const u64 Bn = A ? A << c : 0;
        const int dr = A ? dgb - c : -1;
        A = B;                                          // (a, b) <- (b, a mod b)
        B = Bn;
        dga = dgb;
        dgb = dr;
        u32 y = ma0; ma0 = mb0; mb0 = y;
        y = ma1; ma1 = mb1; mb1 = y;
        dma = dmb;
        dmb = ndm;
        steps++;
    }
    if (steps == 0) {
        L.mode = 1;
        L.k = da - db;
        L.mt[0] = L.mt[1] = L.mt[2] = L.mt[3] = 0;
    } else {
        L.mode = 0;
        L.k = 0;
        L.mt[0] = ma0; L.mt[1] = ma1; L.mt[2] = mb0; L.mt[3] = mb1;
    }
    return L;
}

// lo and hi parts of x (64 bits) times a 32-bit polynomial
GF2E_DEV u64 mul64x32_lo(u64 x, const Masked &m) {
    return clmul_masked(mask32((u32)x), m) ^ (clmul_masked(mask32((u32)(x >> 32)), m) << 32);
}
GF2E_DEV u64 mul64x32_hi(u64 x, const Masked &m) {
    return clmul_masked(mask32((u32)(x >> 32)), m) >> 32;
}
// x * m_a and x * m_b as 96 bits each (lo: bits 0..63, hi: bits 64..95) by
// 16-entry tables T[v] = v * m (v a nibble, entries of up to 35 bits), one
// pass over x's nibbles for both: lookups, shifts and XORs, no multiplies
// (the 32 x 32 -> 64 multiplier of the bit-class product is the apply's
// bottleneck)
GF2E_DEV void mul96_tab2(u64 x, const u64 *Ta, const u64 *Tb, u64 &la, u64 &ha, u64 &lb,
                         u64 &hb) {
    la = ha = lb = hb = 0;
#pragma unroll
    for (int i = 0; i < 16; i++) {
        const unsigned v = (unsigned)(x >> (4 * i)) & 15u;
        const u64 ta = Ta[v], tb = Tb[v];
        la ^= ta << (4 * i);
        lb ^= tb << (4 * i);
        if (i >= 8) {                                  // entries reach bit 34
            ha ^= ta >> (64 - 4 * i);
            hb ^= tb >> (64 - 4 * i);
        }
    }
}
// word w of (X << k) for a vector X
GF2E_DEV u64 shl_word(const u64 *X, long long w, long long k) {
    const long long ks = k >> 6;
    const unsigned kb = (unsigned)(k & 63);
    u64 h = (w >= ks) ? X[w - ks] : 0, l = (w >= ks + 1) ? X[w - ks - 1] : 0;
    return kb ? ((h << kb) | (l >> (64 - kb))) : h;
}
// word w of one new vector / row: mode 0: m0*X + m1*Y; mode 1 (row a): X ^ (Y << k)
GF2E_DEV u64 new_word(int mode, const u64 *X, const u64 *Y, long long w, const Masked &m0,
                      const Masked &m1, long long k, bool is_a) {
    if (mode == 1) return is_a ? (X[w] ^ shl_word(Y, w, k)) : Y[w];
    u64 v = mul64x32_lo(X[w], m0) ^ mul64x32_lo(Y[w], m1);
    if (w >= 1) v ^= mul64x32_hi(X[w - 1], m0) ^ mul64x32_hi(Y[w - 1], m1);
    return v;
}

// (a', b') = M (a, b) with deg a' >= m > deg b'; M written to four arrays of
// mw words (row-major M00 M01 M10 M11).
//
// Lehmer rounds, pipelined: while warps 1..15 apply round r's matrix to the
// vectors A, B and to the accumulated rows (one output word per item, the
// carry from word w-1 recomputed, so no barrier inside the round), warp 0
// computes the three top words of the new A and B itself, reads their
// degrees and 64-bit windows off them and runs round r+1's Euclid steps on
// thread 0.  One barrier per round; when the new windows are not within
// those three words (a large drop in degree), warp 0 scans the new vectors
// after the barrier instead.  Round state is double-buffered by parity.
// Shared memory: V[4][W] (two buffers of A, B), R[2][4][mw].
//
// One CTA per member of a batch (blockIdx.x): member g's operands at
// a + g sa and b + g sb, its matrix at M + g * 4 mw.  A member with db < m
// (db = -1 for one with nothing to do) gets the identity.
struct BaseBatch {
    const u64 *a, *b;
    u64 sa, sb;
    u64 *M;
    long long da[GMAX], db[GMAX], m[GMAX];
};
__global__ void __launch_bounds__(BASE_THREADS)
k_hgcd_base(const BaseBatch BB, u64 W, u64 mw, BaseAcc *acc) {
    const int g = blockIdx.x;
    const u64 *__restrict__ a = BB.a + (u64)g * BB.sa;
    const u64 *__restrict__ b = BB.b + (u64)g * BB.sb;
    const long long da0 = BB.da[g], db0 = BB.db[g], m = BB.m[g];
    u64 *__restrict__ Mout = BB.M + (u64)g * 4 * mw;
    extern __shared__ u64 sh[];
    u64 *V = sh;
    u64 *R = sh + 4 * W;
    __shared__ int s_va[2], s_vb[2], s_ra[2], s_mode[2], s_done[2], s_slow;
    __shared__ long long s_k[2], s_top[2], s_md[2];
    __shared__ u32 s_m[2][4];
    __shared__ u64 s_tab[(BASE_THREADS / 32 / 4) * 3][64];   // per apply warp: v * m_e
    const int tid = threadIdx.x;
    for (u64 i = tid; i < 4 * W; i += BASE_THREADS) {
        u64 v = 0;
        if (i < W) v = (i <= (u64)(da0 >> 6)) ? a[i] : 0;
        else if (i < 2 * W) { u64 j = i - W; v = (db0 >= 0 && j <= (u64)(db0 >> 6)) ? b[j] : 0; }
        V[i] = v;
    }
    for (u64 i = tid; i < 8 * mw; i += BASE_THREADS) R[i] = (i == 0 || i == 3 * mw) ? 1 : 0;
    __syncthreads();
    const long long max_rounds = 2 * (da0 + 2) + 16;
    int status = GF2E_OK;
    long long rounds = 0;
    const long long cyc0 = clock64();
    long long cyc_serial = 0;

    // thread 0: publish round q's state from degrees/roles and windows
    auto publish = [&](int q, int va, int vb, int ra, long long da, long long db, u64 wa, u64 wb,
                       long long md, long long round) {
        if (da < db) {
            int x = va; va = vb; vb = x;
            ra ^= 1;
            long long t = da; da = db; db = t;
            u64 u = wa; wa = wb; wb = u;
        }
        s_va[q] = va; s_vb[q] = vb; s_ra[q] = ra;
        s_top[q] = da >> 6;
        s_md[q] = md;
        if (db < m || round > max_rounds) {
            s_done[q] = 1;
            if (round > max_rounds) status = GF2E_ERR_TIMEOUT;
            rounds = round;
            return;
        }
        s_done[q] = 0;
        const long long lo = da >= 63 ? da - 63 : 0;
        const long long c0 = clock64();
        Lehmer L = lehmer_round(wa, wb, da, db, lo, m);
        cyc_serial += clock64() - c0;
        s_mode[q] = L.mode;
        s_k[q] = L.k;
        for (int i = 0; i < 4; i++) s_m[q][i] = L.mt[i];
    };
    // thread 0: degrees and windows of vectors va, vb read from shared memory
    auto publish_from_vectors = [&](int q, int va, int vb, int ra, long long da, long long db,
                                    long long md, long long round) {
        const long long dhi = max(da, db);
        const long long lo = dhi >= 63 ? dhi - 63 : 0;
        publish(q, va, vb, ra, da, db, win_at(V + (u64)va * W, (long long)W, lo),
                win_at(V + (u64)vb * W, (long long)W, lo), md, round);
    };
    if (tid == 0) publish_from_vectors(0, 0, 1, 0, da0, db0, 0, 0);
    __syncthreads();

    long long final_round = 0;
    for (long long round = 0;; round++) {
        const int p = (int)(round & 1), q = p ^ 1;
        if (s_done[p]) { final_round = round; break; }
        const int va = s_va[p], vb = s_vb[p], ra = s_ra[p], mode = s_mode[p];
        const long long top = s_top[p], md = s_md[p], k = s_k[p];
        // live words: vectors 0..top; rows 0..nwm (the growth of this round included)
        const long long nwv = top + 1;
        const long long nwm = min((long long)mw - 1, md + (mode == 1 ? (k >> 6) + 1 : 1));
        int spare[2], ns = 0;
        for (int i = 0; i < 4 && ns < 2; i++)
            if (i != va && i != vb) spare[ns++] = i;
        const u64 *A = V + (u64)va * W, *B = V + (u64)vb * W;
        u64 *A2 = V + (u64)spare[0] * W, *B2 = V + (u64)spare[1] * W;
        const u64 *RA = R + (u64)(p * 4 + 2 * ra) * mw, *RB = R + (u64)(p * 4 + 2 * (ra ^ 1)) * mw;
        u64 *N = R + (u64)q * 4 * mw;
        const Masked m0 = mask32(s_m[p][0]), m1 = mask32(s_m[p][1]), m2 = mask32(s_m[p][2]),
                     m3 = mask32(s_m[p][3]);
        const long long md_next = min((long long)mw - 2, md + (mode == 1 ? (k >> 6) + 1 : 1));
        const int warp = tid >> 5;
        if (warp != 0 && (warp & 3) != 0) {
            // the apply runs on the warps of the other three schedulers, so
            // warp 0's serial chain keeps its scheduler (warp w is on w % 4).
            // Work in chunks of 31 output words of one pair of outputs: the
            // new vectors (A', B') from (A, B), or the new row entries
            // (N[col], N[2 + col]) from (RA[col], RB[col]).  Lane l takes
            // word 31 c + l - 1 of the inputs, computes its full products
            // (by the warp's nibble tables of the four matrix entries) and
            // passes their high words up one lane: lane 0's word only feeds
            // lane 1, so every input word is multiplied once.
            constexpr int APPLY_WARPS = (BASE_THREADS / 32 / 4) * 3;
            const int aw = warp - 1 - (warp >> 2), lane = tid & 31;
            u64 *T = s_tab[aw];                         // T[16 e + v] = v * m_e
            if (mode != 1) {
                for (int i = lane; i < 64; i += 32) {
                    const u64 me = s_m[p][i >> 4];
                    u64 t = 0;
#pragma unroll
                    for (int b = 0; b < 4; b++)
                        if ((i >> b) & 1) t ^= me << b;
                    T[i] = t;
                }
                __syncwarp();
            }
            const long long ncv = (nwv + 30) / 31, ncr = (nwm + 31) / 31;
            for (long long c = aw; c < ncv + 2 * ncr; c += APPLY_WARPS) {
                const bool vec = c < ncv;
                const long long cr = c - ncv;
                const int col = vec ? 0 : (int)(cr / ncr);
                const long long n = vec ? nwv : nwm + 1;
                const long long w = 31 * (vec ? c : cr - col * ncr) + lane - 1;
                const u64 *X = vec ? A : RA + (u64)col * mw, *Y = vec ? B : RB + (u64)col * mw;
                u64 *O0 = vec ? A2 : N + (u64)col * mw, *O1 = vec ? B2 : N + (u64)(2 + col) * mw;
                const bool in = w >= 0 && w < n;
                u64 o0 = 0, o1 = 0;
                if (mode == 1) {                        // (X ^ (Y << k), Y)
                    if (in) {
                        o0 = X[w] ^ shl_word(Y, w, k);
                        o1 = Y[w];
                    }
                } else {                                // (m0 X + m1 Y, m2 X + m3 Y)
                    u64 l0, h0, l1, h1, tl0, th0, tl1, th1;
                    mul96_tab2(in ? X[w] : 0, T, T + 32, l0, h0, l1, h1);        // x m0, x m2
                    mul96_tab2(in ? Y[w] : 0, T + 16, T + 48, tl0, th0, tl1, th1);  // y m1, y m3
                    l0 ^= tl0; h0 ^= th0;
                    l1 ^= tl1; h1 ^= th1;
                    o0 = l0 ^ __shfl_up_sync(0xffffffffu, h0, 1);
                    o1 = l1 ^ __shfl_up_sync(0xffffffffu, h1, 1);
                }
                if (lane >= 1 && in) {
                    O0[w] = o0;
                    O1[w] = o1;
                }
            }
            // stale words of the new vectors above the live range
            constexpr int APPLY_THREADS = APPLY_WARPS * 32;
            const int at = aw * 32 + lane;
            for (long long w = nwv + at; w < (long long)W; w += APPLY_THREADS) {
                A2[w] = 0;
                B2[w] = 0;
            }
        } else if (warp == 0) {
            // warp 0: the three top words of the new A (lanes 0-2) and B (3-5)
            // in one pass (each lane with its own matrix row), then their
            // degrees and the next windows by ballot and shuffle
            const int lane = tid;
            const bool vb = lane >= 3;
            const long long w = top - (lane % 3);
            u64 val = 0;
            if (lane < 6 && w >= 0)
                val = new_word(mode, A, B, w, vb ? m2 : m0, vb ? m3 : m1, k, !vb);
            const unsigned nz = __ballot_sync(0xffffffffu, lane < 6 && val != 0);
            const int fa = __ffs(nz & 7u) - 1, fb = __ffs((nz >> 3) & 7u) - 1;
            const u64 ta = __shfl_sync(0xffffffffu, val, fa < 0 ? 0 : fa);
            const u64 tb = __shfl_sync(0xffffffffu, val, fb < 0 ? 3 : 3 + fb);
            const long long dn0 = fa < 0 ? -1 : (top - fa) * 64 + 63 - __clzll(ta);
            const long long dn1 = fb < 0 ? -1 : (top - fb) * 64 + 63 - __clzll(tb);
            bool slow = dn0 < 0 || dn1 < 0;
            long long lo = 0;
            if (!slow) {
                const long long dhi = max(dn0, dn1);
                lo = dhi >= 63 ? dhi - 63 : 0;
                slow = (lo >> 6) < top - 2;
            }
            // the windows' low words are words lo/64 (lane top - lo/64) and
            // lo/64 + 1 (one lane lower) of the new vectors
            const int ia = slow ? 0 : (int)(top - (lo >> 6));
            const int ib = ia >= 1 ? ia - 1 : 0;
            const u64 x0a = __shfl_sync(0xffffffffu, val, ia), x1a = __shfl_sync(0xffffffffu, val, ib);
            const u64 x0b = __shfl_sync(0xffffffffu, val, 3 + ia), x1b = __shfl_sync(0xffffffffu, val, 3 + ib);
            if (lane == 0) {
                if (!slow) {
                    const unsigned sb = (unsigned)(lo & 63);
                    publish(q, spare[0], spare[1], 0, dn0, dn1, funnel64(x0a, ia >= 1 ? x1a : 0, sb),
                            funnel64(x0b, ia >= 1 ? x1b : 0, sb), md_next, round + 1);
                }
                s_slow = slow;
            }
        }
        __syncthreads();
        if (s_slow) {                                  // degrees from the full new vectors
            if (tid < 32) {
                const long long d0 = warp_degree(A2, top), d1 = warp_degree(B2, top);
                if (tid == 0) publish_from_vectors(q, spare[0], spare[1], 0, d0, d1, md_next, round + 1);
            }
            __syncthreads();
        }
    }
    // matrix out, rows in (A, B) order; the final round's parity holds them
    const int pf = (int)(final_round & 1);
    __syncthreads();
    const int fra = s_ra[pf];
    for (u64 w = tid; w < 2 * mw; w += BASE_THREADS) {
        Mout[w] = R[(u64)(pf * 4 + 2 * fra) * mw + w];
        Mout[2 * mw + w] = R[(u64)(pf * 4 + 2 * (fra ^ 1)) * mw + w];
    }
    if (tid == 0) {
        atomicAdd(&acc->rounds, (unsigned long long)rounds);
        atomicAdd(&acc->cyc_serial, (unsigned long long)cyc_serial);
        atomicAdd(&acc->cyc_total, (unsigned long long)(clock64() - cyc0));
        if (status != GF2E_OK) atomicCAS(&acc->worst, GF2E_OK, status);
    }
}

// ------------------------------------------------------------------ host
struct Fail {
    int st;
};
inline void ck(int st) {
    if (st != GF2E_OK) throw Fail{st};
}
inline void ckc(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw Fail{gf2e::cuda_status(e, what)};
}

struct Pool {
    cudaMemPool_t pool = nullptr;
};

// Sub-allocator for one gcd's device buffers.  Every buffer of a gcd is used
// on that gcd's stream only, so a block given back can go to the next
// request at once: stream order keeps the kernels that used it ahead of the
// next user, as cudaFreeAsync would, without an allocator call per buffer
// (a half-gcd at r = 136279841 makes several hundred thousand buffers, and
// concurrent gcds would otherwise queue on those calls).  Blocks are powers
// of two words, carved from chunks taken from the stream-ordered pool and
// kept on per-size free lists; the chunks go back to the pool at the end.
class Arena {
public:
    Arena(cudaStream_t st, cudaMemPool_t pool) : st_(st), pool_(pool) {}
    ~Arena() {
        for (u64 *c : chunks_) cudaFreeAsync(c, st_);
    }
    Arena(const Arena &) = delete;
    Arena &operator=(const Arena &) = delete;

    // size classes 2^e (1 + j/4), j = 0..3, e >= 6: a block wastes under a
    // fifth of its size (lockstep batches make single buffers of GBs)
    static size_t class_words(int cls) {
        const int e = cls >> 2, j = cls & 3;
        return ((size_t)1 << e) + (size_t)j * ((size_t)1 << (e - 2));
    }
    static int class_of(size_t words) {
        int e = 6;
        while (((size_t)1 << (e + 1)) < words) e++;
        int cls = 4 * e;
        while (class_words(cls) < words) cls++;
        return cls;
    }
    u64 *get(size_t words, int &cls) {
        cls = class_of(words);
        if (!free_[cls].empty()) {
            u64 *p = free_[cls].back();
            free_[cls].pop_back();
            return p;
        }
        const size_t need = class_words(cls);
        if (left_ < need) {
            const size_t chunk = std::max(need, (size_t)1 << 22);    // 32 MB or the block
            void *c = nullptr;
            const cudaError_t e = cudaMallocFromPoolAsync(&c, chunk * 8, pool_, st_);
            if (e == cudaErrorMemoryAllocation) {      // not sticky: the caller may retry smaller
                cudaGetLastError();
                gf2e::set_error("hgcd pool allocation: out of device memory");
                throw Fail{GF2E_ERR_NOMEM};
            }
            ckc_arena(e);
            chunks_.push_back((u64 *)c);
            cur_ = (u64 *)c;
            left_ = chunk;
        }
        u64 *p = cur_;
        cur_ += need;
        left_ -= need;
        return p;
    }
    void put(u64 *p, int cls) { free_[cls].push_back(p); }

private:
    static void ckc_arena(cudaError_t e) { ckc(e, "hgcd pool allocation"); }
    cudaStream_t st_;
    cudaMemPool_t pool_;
    std::vector<u64 *> chunks_;
    std::vector<u64 *> free_[4 * 64];
    u64 *cur_ = nullptr;
    size_t left_ = 0;
};

// device buffer from the gcd's arena, given back when the last owner drops it
struct DBuf {
    u64 *p = nullptr;
    size_t words = 0;
    cudaStream_t st = nullptr;
    Arena *arena = nullptr;
    int cls = 0;
    virtual ~DBuf() {
        if (p && arena) arena->put(p, cls);
    }
};
typedef std::shared_ptr<DBuf> Buf;

// a view into another buffer that keeps it alive
Buf view_of(const Buf &owner, size_t off, size_t words) {
    struct View : DBuf {
        Buf keep;
        ~View() { p = nullptr; }
    };
    auto v = std::make_shared<View>();
    v->keep = owner;
    v->p = owner->p + off;
    v->words = words;
    v->st = owner->st;
    return v;
}

// the base kernel's dynamic shared memory limit, raised once per device
void base_smem_attr() {
    static std::mutex mu;
    static bool attr[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    if (dev >= 0 && dev < 64 && !attr[dev]) {
        ckc(cudaFuncSetAttribute(k_hgcd_base, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 200 * 1024), "k_hgcd_base smem attribute");
        attr[dev] = true;
    }
}

struct Tunables {
    long long base_bits = 1 << 14;       // n <= base_bits: one-CTA base kernel
    long long fft_bits = 1 << 19;        // products above this many bits use the FFT
    long long small_gcd_bits = 1 << 15;  // finish with the quadratic gcd below this
    int streams = 2;                     // lockstep batches run at once
};

// A lockstep batch fills the GPU with every product, so the FFT's lower
// work pays from smaller sizes than for one gcd, whose small products leave
// most SMs idle either way (measured, 64 gcds of 16 Mbit at once: 6.3 s
// with the FFT from 2^15 bits, 6.5 s from 2^16, 7.5 s from 2^17, 8.3 s from
// 2^18, 11.7 s from 2^19, 17.2 s from 2^20).
Tunables tunables(bool lockstep = false) {
    Tunables t;
    if (lockstep) t.fft_bits = 1 << 16;
    if (const char *e = getenv("GF2E_HGCD_BASE_BITS")) t.base_bits = atoll(e);
    if (const char *e = getenv("GF2E_HGCD_FFT_BITS")) t.fft_bits = atoll(e);
    if (const char *e = getenv("GF2E_HGCD_SMALL_BITS")) t.small_gcd_bits = atoll(e);
    if (const char *e = getenv("GF2E_HGCD_STREAMS")) t.streams = std::max(1, atoi(e));
    t.base_bits = std::max(256LL, std::min(t.base_bits, 1LL << 16));
    t.small_gcd_bits = std::max(t.small_gcd_bits, 2 * t.base_bits);
    return t;
}

struct Stats {
    long long nodes = 0, bases = 0, base_rounds = 0, fft_mul2 = 0, school_mul2 = 0, divsteps = 0,
              probes = 0, cyc_serial = 0, cyc_total = 0;
    double us_base = 0, us_products = 0, us_division = 0, us_small = 0;
};

// adds the wall time of a scope to a counter
struct Timer {
    double &acc;
    std::chrono::steady_clock::time_point t0;
    explicit Timer(double &a) : acc(a), t0(std::chrono::steady_clock::now()) {}
    ~Timer() {
        acc += std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count();
    }
};

// ================================================================ lockstep
// A batch of G gcds (G <= GMAX) stepped through the half-gcd recursion
// together, driven by one host thread on one stream.  The members' sizes
// differ by a few bits at every node (the degree drops are data-dependent),
// so every launch serves all members with their own degrees and shifts,
// and the host takes every decision per member:
//   * a member is active at a node while deg b >= m for it; inactive
//     members get the identity matrix there (the base kernel writes it, and
//     every product with it is exact), so the composition stays correct;
//   * the node recurses while its largest active member is above the base
//     size, so all members take the same path through the tree;
//   * degree reads (probes), division steps and the final quadratic gcds
//     are one call for all members.
// Launches and host round trips per gcd fall by the batch size, and the
// base cases run as one grid of G CTAs.
typedef std::vector<char> Mask;

bool any_of(const Mask &m) {
    for (char c : m)
        if (c) return true;
    return false;
}
bool all_of(const Mask &m) {
    for (char c : m)
        if (!c) return false;
    return true;
}
unsigned long long mask_bits(const Mask &m) {
    unsigned long long b = 0;
    for (size_t g = 0; g < m.size(); g++)
        if (m[g]) b |= 1ull << g;
    return b;
}

// member g at base() + g * stride; deg exact for remainders, a bound for
// matrix entries (words(g) covers every nonzero word either way)
struct BPoly {
    Buf b;
    u64 stride = 0;
    std::vector<long long> deg;
    std::vector<u64> win;          // top 64 bits at deg, valid after a probe of g
    bool has_win = false;          // every member's window valid
    u64 *base() const { return b ? b->p : nullptr; }
    u64 words(int g) const { return deg[g] < 0 ? 0 : (u64)(deg[g] >> 6) + 1; }
};
struct BMat {
    BPoly e[4];                    // M00 M01 M10 M11
    bool ident = false;            // the identity for every member
};

class HgcdBatch {
public:
    HgcdBatch(int G, cudaStream_t st, cudaMemPool_t pool)
        : arena_(st, pool), G_(G), st_(st), tn_(tunables(G > 1)) {
        d_probe_ = alloc(GMAX * 8);
        d_res_ = alloc(8);
        ckc(cudaMemsetAsync(d_res_->p, 0, sizeof(BaseAcc), st_), "hgcd base accumulator");
        // last: a constructor that throws runs no destructor
        ckc(cudaMallocHost(&h_probe_, (size_t)GMAX * 8 * sizeof(long long)), "hgcd probe host buffer");
    }
    ~HgcdBatch() {
        if (h_probe_) cudaFreeHost(h_probe_);
    }
    HgcdBatch(const HgcdBatch &) = delete;
    HgcdBatch &operator=(const HgcdBatch &) = delete;
    Stats stats;

    // gcd of every job's operands; deg_out[g] as gf2e_gcd_large, the gcd
    // copied to the job's g_dev where it fits
    void run(const gf2e_gcd_job *jobs, int64_t *deg_out) {
        BPoly a = load(jobs, true), b = load(jobs, false);
        Mask done(G_, 0), small(G_, 0);
        BPoly sg;                                  // results of the quadratic gcds
        sg.stride = 1;
        sg.deg.assign(G_, -1);
        std::vector<Buf> small_keep;
        std::vector<u64 *> small_ptr(G_, nullptr);
        for (long long it = 0;; it++) {
            if (it > 4 * 64 + 64) throw Fail{gf2e::invalid("hgcd batch: no convergence")};
            Mask sw(G_, 0), fin(G_, 0);
            for (int g = 0; g < G_; g++) sw[g] = !done[g] && a.deg[g] < b.deg[g];
            if (any_of(sw)) swap_members(sw, a, b);
            for (int g = 0; g < G_; g++)
                if (!done[g] && b.deg[g] < 0) done[g] = 1;        // gcd = a
            for (int g = 0; g < G_; g++)
                fin[g] = !done[g] && a.deg[g] < tn_.small_gcd_bits;
            if (any_of(fin)) {
                small_gcds(a, b, fin, sg, small_keep, small_ptr);
                for (int g = 0; g < G_; g++)
                    if (fin[g]) { done[g] = 1; small[g] = 1; }
            }
            if (all_of(done)) break;
            Mask eq(G_, 0), act(G_, 0);
            for (int g = 0; g < G_; g++) eq[g] = !done[g] && a.deg[g] == b.deg[g];
            if (any_of(eq)) {
                divstep(a, b, nullptr, eq);
                continue;
            }
            for (int g = 0; g < G_; g++) act[g] = !done[g];
            BMat M = hgcd(a, b, act);
            if (!M.ident) {
                BPoly c, d;
                mat_vec(M, a, b, c, d);
                a = c;
                b = d;
            }
            for (int g = 0; g < G_; g++) sw[g] = act[g] && a.deg[g] < b.deg[g];
            if (any_of(sw)) swap_members(sw, a, b);
            Mask dv(G_, 0);
            for (int g = 0; g < G_; g++) dv[g] = act[g] && b.deg[g] >= 0;
            if (any_of(dv)) divstep(a, b, nullptr, dv);
        }
        finish_bases();
        for (int g = 0; g < G_; g++) {
            const long long d = small[g] ? sg.deg[g] : a.deg[g];
            const u64 *src = small[g] ? small_ptr[g] : a.base() + (u64)g * a.stride;
            deg_out[g] = d < 0 ? 0 : d;
            const gf2e_gcd_job &j = jobs[g];
            if (j.g_dev && j.g_cap_words) {
                const u64 gw = d < 0 ? 0 : (u64)(d >> 6) + 1;
                if (gw <= j.g_cap_words) {
                    ckc(cudaMemsetAsync(j.g_dev, 0, j.g_cap_words * 8, st_), "gcd out clear");
                    if (gw) ckc(cudaMemcpyAsync(j.g_dev, src, gw * 8, cudaMemcpyDeviceToDevice, st_),
                                "gcd out");
                }
            }
        }
        ckc(cudaStreamSynchronize(st_), "hgcd batch done");
    }

private:
    Buf alloc(size_t words) {
        auto b = std::make_shared<DBuf>();
        b->st = st_;
        b->words = std::max<size_t>(words, 1);
        b->p = arena_.get(b->words, b->cls);
        b->arena = &arena_;
        return b;
    }
    BPoly make(u64 stride, bool zero) {
        BPoly r;
        r.stride = std::max<u64>(stride, 1);
        r.b = alloc((size_t)G_ * r.stride);
        r.deg.assign(G_, -1);
        r.win.assign(G_, 0);
        if (zero) ckc(cudaMemsetAsync(r.base(), 0, (size_t)G_ * r.stride * 8, st_), "hgcd memset");
        return r;
    }
    BPoly load(const gf2e_gcd_job *jobs, bool first) {
        u64 stride = 1;
        for (int g = 0; g < G_; g++) {
            const u64 bits = first ? jobs[g].abits : jobs[g].bbits;
            stride = std::max<u64>(stride, (bits + 63) / 64 + 1);
        }
        BPoly r = make(stride, true);
        for (int g = 0; g < G_; g++) {
            const u64 bits = first ? jobs[g].abits : jobs[g].bbits;
            const u64 *src = first ? jobs[g].a_dev : jobs[g].b_dev;
            const u64 nw = (bits + 63) / 64;
            if (nw) ckc(cudaMemcpyAsync(r.base() + (u64)g * stride, src, nw * 8,
                                        cudaMemcpyDeviceToDevice, st_), "hgcd load");
            r.deg[g] = (long long)nw * 64 - 1;      // bound until probed
        }
        probe({&r}, nullptr);
        return r;
    }

    // exact degrees and windows of up to four batched polynomials whose deg
    // is an upper bound, for the members in `which` (all when null)
    void probe(std::initializer_list<BPoly *> ps, const Mask *which) {
        ProbeBatch P;
        memset(&P, 0, sizeof P);
        int n = 0;
        for (BPoly *p : ps) {
            P.p[n] = p->base();
            P.stride[n] = p->stride;
            for (int g = 0; g < G_; g++)
                P.nw[n][g] = (!which || (*which)[g]) ? (u32)p->words(g) : 0;
            n++;
        }
        k_probe_b<<<G_, 32 * n, 0, st_>>>(P, n, (long long *)d_probe_->p);
        ckc(cudaGetLastError(), "k_probe_b");
        ckc(cudaMemcpyAsync(h_probe_, d_probe_->p, (size_t)G_ * 8 * sizeof(long long),
                            cudaMemcpyDeviceToHost, st_), "probe read");
        ckc(cudaStreamSynchronize(st_), "probe sync");
        stats.probes++;
        int i = 0;
        for (BPoly *p : ps) {
            for (int g = 0; g < G_; g++)
                if (!which || (*which)[g]) {
                    p->deg[g] = h_probe_[(g * 4 + i) * 2];
                    p->win[g] = (u64)h_probe_[(g * 4 + i) * 2 + 1];
                }
            p->has_win = !which;
            i++;
        }
    }

    // member slices x quo x^k[g] for the members in `which`, zero for the rest
    BPoly shr(const BPoly &x, const std::vector<long long> &k, const Mask &which) {
        BPoly r;
        r.deg.assign(G_, -1);
        r.win.assign(G_, 0);
        u64 stride = 1;
        for (int g = 0; g < G_; g++)
            if (which[g] && x.deg[g] >= k[g]) {
                r.deg[g] = x.deg[g] - k[g];
                stride = std::max(stride, r.words(g));
            }
        r.stride = stride;
        r.b = alloc((size_t)G_ * stride);
        ShrBatch B;
        memset(&B, 0, sizeof B);
        B.src = x.base();
        B.ss = x.stride;
        B.dst = r.base();
        B.ds = stride;
        for (int g = 0; g < G_; g++) {
            B.k[g] = (u64)std::max(0LL, k[g]);
            B.ns[g] = (u32)x.words(g);
            B.nd[g] = (u32)r.words(g);
        }
        k_shr_b<<<dim3(std::max(1, gf2e::grid_for(stride, 256) / G_ + 1), G_), 256, 0, st_>>>(B);
        ckc(cudaGetLastError(), "k_shr_b");
        return r;
    }

    // member slices (bit g of sel) ? t : f
    BPoly select(const Mask &sel, const BPoly &t, const BPoly &f) {
        BPoly r;
        r.deg.assign(G_, -1);
        r.win.assign(G_, 0);
        u64 stride = 1;
        for (int g = 0; g < G_; g++) {
            const BPoly &src = sel[g] ? t : f;
            r.deg[g] = src.deg[g];
            r.win[g] = src.win[g];
            stride = std::max(stride, src.words(g));
        }
        r.stride = stride;
        r.b = alloc((size_t)G_ * stride);
        SelectBatch B;
        memset(&B, 0, sizeof B);
        B.t = t.base();
        B.f = f.base();
        B.out = r.base();
        B.st = t.stride;
        B.sf = f.stride;
        B.so = stride;
        B.mask = mask_bits(sel);
        for (int g = 0; g < G_; g++) {
            B.nt[g] = (u32)t.words(g);
            B.nf[g] = (u32)f.words(g);
        }
        k_select_b<<<dim3(std::max(1, gf2e::grid_for(stride, 256) / G_ + 1), G_), 256, 0, st_>>>(B);
        ckc(cudaGetLastError(), "k_select_b");
        r.has_win = t.has_win && f.has_win;
        return r;
    }
    void swap_members(const Mask &sw, BPoly &a, BPoly &b) {
        if (all_of(sw)) {
            std::swap(a, b);
            return;
        }
        BPoly na = select(sw, b, a), nb = select(sw, a, b);
        a = na;
        b = nb;
    }

    BMat identity() {
        BMat I;
        I.ident = true;
        return I;
    }
    BMat materialize(const BMat &M) {
        if (!M.ident) return M;
        BMat r;
        for (int i = 0; i < 4; i++) {
            r.e[i] = make(1, true);
            if (i == 0 || i == 3) {
                k_set_one_b<<<(G_ + 63) / 64, 64, 0, st_>>>(r.e[i].base(), 1, G_);
                ckc(cudaGetLastError(), "k_set_one_b");
                r.e[i].deg.assign(G_, 0);
            }
        }
        return r;
    }

    // up to four sums x1*y1 + x2*y2 (schoolbook, one zeroed buffer); the
    // result degrees are bounds
    struct PairB {
        const BPoly *x1, *y1, *x2, *y2;
    };
    void mul2_school(const PairB *jobs, int nj, BPoly *outs) {
        Mul2Batch J;
        memset(&J, 0, sizeof J);
        u64 off[4], total = 0, nmax = 0, xmax = 0;
        std::vector<long long> dm[4];
        for (int z = 0; z < nj; z++) {
            const PairB &P = jobs[z];
            dm[z].assign(G_, -1);
            J.x1[z] = P.x1->base(); J.sx1[z] = P.x1->stride;
            J.y1[z] = P.y1->base(); J.sy1[z] = P.y1->stride;
            if (P.x2) {
                J.x2[z] = P.x2->base(); J.sx2[z] = P.x2->stride;
                J.y2[z] = P.y2->base(); J.sy2[z] = P.y2->stride;
            }
            u64 so = 1;
            for (int g = 0; g < G_; g++) {
                const bool t1 = P.x1->deg[g] >= 0 && P.y1->deg[g] >= 0;
                const bool t2 = P.x2 && P.x2->deg[g] >= 0 && P.y2->deg[g] >= 0;
                long long d = -1;
                if (t1) d = std::max(d, P.x1->deg[g] + P.y1->deg[g]);
                if (t2) d = std::max(d, P.x2->deg[g] + P.y2->deg[g]);
                dm[z][g] = d;
                const u64 nout = d < 0 ? 1 : (u64)(d >> 6) + 2;
                J.nout[z][g] = (u32)nout;
                so = std::max(so, nout);
                if (t1) { J.nx1[z][g] = (u32)P.x1->words(g); J.ny1[z][g] = (u32)P.y1->words(g); }
                if (t2) { J.nx2[z][g] = (u32)P.x2->words(g); J.ny2[z][g] = (u32)P.y2->words(g); }
                xmax = std::max<u64>(xmax, std::max(J.nx1[z][g], J.nx2[z][g]));
            }
            J.so[z] = so;
            off[z] = total;
            total += so * G_;
            nmax = std::max(nmax, so);
        }
        Buf all = alloc(total);
        ckc(cudaMemsetAsync(all->p, 0, total * 8, st_), "hgcd memset");
        for (int z = 0; z < nj; z++) {
            J.out[z] = (unsigned long long *)(all->p + off[z]);
            outs[z] = BPoly();
            outs[z].b = view_of(all, off[z], J.so[z] * G_);
            outs[z].stride = J.so[z];
            outs[z].deg = dm[z];
            outs[z].win.assign(G_, 0);
        }
        const u64 chunk = 32;
        dim3 grid((unsigned)((nmax / 2 + 1 + 127) / 128), (unsigned)std::max<u64>(1, (xmax + chunk - 1) / chunk),
                  (unsigned)(nj * G_));
        k_mul2_b<<<grid, 128, 0, st_>>>(J, G_, chunk);
        ckc(cudaGetLastError(), "k_mul2_b");
        stats.school_mul2 += nj;
    }

    static u64 chunks(const BPoly &p, int g) {
        return p.deg[g] < 0 ? 0 : ((u64)p.deg[g] + 1 + 31) / 32;
    }
    static u64 max_chunks(const BPoly &p) {
        u64 c = 0;
        for (size_t g = 0; g < p.deg.size(); g++) c = std::max(c, chunks(p, (int)g));
        return c;
    }
    // forward transforms of every member of p into f (G x n)
    void fwd(gf2e_fft_plan *plan, const BPoly &p, u64 *f, u64 n) {
        const u64 nch = max_chunks(p);
        if (!nch) ckc(cudaMemsetAsync(f, 0, (size_t)G_ * n * 8, st_), "fft zero operand");
        else ck(gf2e::fft_fwd_packed_batch(plan, f, n, reinterpret_cast<const u32 *>(p.base()),
                                           2 * p.stride, nch, 0, G_, st_));
    }
    // o <- inverse of X1 Y1 + X2 Y2 (pointwise), overlap-added into a new
    // batched polynomial of degree bounds dm
    BPoly product_out(gf2e_fft_plan *plan, u64 *o, const u64 *x1, const u64 *y1, const u64 *x2,
                      const u64 *y2, u64 n, u64 need, const std::vector<long long> &dm) {
        const u64 tot = (u64)G_ * n;
        k_pw_muladd<<<gf2e::grid_for(tot, 256), 256, 0, st_>>>(o, x1, y1, x2, y2, tot);
        ckc(cudaGetLastError(), "k_pw_muladd");
        ck(gf2e::fft_run_batch(plan, false, o, n, G_, st_));
        u64 so = 1;
        for (int g = 0; g < G_; g++)
            if (dm[g] >= 0) so = std::max(so, (u64)(dm[g] >> 6) + 2);
        BPoly out = make(so, false);
        ck(gf2e::overlap_add_batch(o, n, need, out.base(), so, so, G_, st_));
        for (int g = 0; g < G_; g++) out.deg[g] = dm[g] < 0 ? -1 : std::min<long long>(dm[g], (long long)so * 64 - 1);
        return out;
    }

    // (c, d) = M (a, b); exact degrees
    void mat_vec(const BMat &M, const BPoly &a, const BPoly &b, BPoly &c, BPoly &d) {
        Timer tm(stats.us_products);
        if (M.ident) {
            c = a;
            d = b;
            return;
        }
        long long dmax = -1;
        for (int g = 0; g < G_; g++)
            for (int i = 0; i < 4; i++) {
                const BPoly &v = (i & 1) ? b : a;
                if (M.e[i].deg[g] >= 0 && v.deg[g] >= 0) dmax = std::max(dmax, M.e[i].deg[g] + v.deg[g]);
            }
        if (dmax + 1 > tn_.fft_bits) {
            fft_mat_vec(M, a, b, c, d);
        } else {
            PairB P[2] = {{&M.e[0], &a, &M.e[1], &b}, {&M.e[2], &a, &M.e[3], &b}};
            BPoly o[2];
            mul2_school(P, 2, o);
            c = o[0];
            d = o[1];
        }
        probe({&c, &d}, nullptr);
    }

    std::vector<long long> sum_bound(const BPoly &x1, const BPoly &y1, const BPoly &x2,
                                     const BPoly &y2) {
        std::vector<long long> dm(G_, -1);
        for (int g = 0; g < G_; g++) {
            if (x1.deg[g] >= 0 && y1.deg[g] >= 0) dm[g] = std::max(dm[g], x1.deg[g] + y1.deg[g]);
            if (x2.deg[g] >= 0 && y2.deg[g] >= 0) dm[g] = std::max(dm[g], x2.deg[g] + y2.deg[g]);
        }
        return dm;
    }
    static int fft_m(u64 need) {
        int m = 1;
        while (((u64)1 << m) < need) m++;
        return m;
    }

    void fft_mat_vec(const BMat &M, const BPoly &a, const BPoly &b, BPoly &c, BPoly &d) {
        u64 need = 1;
        for (int g = 0; g < G_; g++)
            for (int i = 0; i < 4; i++) {
                const BPoly &v = (i & 1) ? b : a;
                if (M.e[i].deg[g] >= 0 && v.deg[g] >= 0)
                    need = std::max(need, chunks(M.e[i], g) + chunks(v, g) - 1);
            }
        gf2e_fft_plan *plan = gf2e::cached_plan(fft_m(need));
        if (!plan) throw Fail{GF2E_ERR_CUDA};
        const u64 n = gf2e::fft_plan_n(plan);
        Buf Fa = alloc(G_ * n), Fb = alloc(G_ * n);
        fwd(plan, a, Fa->p, n);
        fwd(plan, b, Fb->p, n);
        for (int row = 0; row < 2; row++) {     // one row's transforms live at a time
            Buf F0 = alloc(G_ * n), F1 = alloc(G_ * n);
            fwd(plan, M.e[2 * row], F0->p, n);
            fwd(plan, M.e[2 * row + 1], F1->p, n);
            (row ? d : c) = product_out(plan, F0->p, F0->p, Fa->p, F1->p, Fb->p, n, need,
                                        sum_bound(M.e[2 * row], a, M.e[2 * row + 1], b));
        }
        stats.fft_mul2 += 2;
    }

    // M2 * M1 (degree bounds)
    BMat mat_mul(const BMat &M2, const BMat &M1) {
        Timer tm(stats.us_products);
        if (M2.ident) return M1;
        if (M1.ident) return M2;
        long long dmax = 0;
        for (int g = 0; g < G_; g++)
            for (int i = 0; i < 2; i++)
                for (int j = 0; j < 2; j++)
                    dmax = std::max(dmax, std::max(M2.e[2 * i].deg[g] + M1.e[j].deg[g],
                                                   M2.e[2 * i + 1].deg[g] + M1.e[2 + j].deg[g]));
        BMat r;
        if (dmax + 1 > tn_.fft_bits) {
            u64 need = 1;
            for (int g = 0; g < G_; g++)
                for (int i = 0; i < 2; i++)
                    for (int j = 0; j < 2; j++)
                        for (int k = 0; k < 2; k++) {
                            const BPoly &x = M2.e[2 * i + k], &y = M1.e[2 * k + j];
                            if (x.deg[g] >= 0 && y.deg[g] >= 0)
                                need = std::max(need, chunks(x, g) + chunks(y, g) - 1);
                        }
            gf2e_fft_plan *plan = gf2e::cached_plan(fft_m(need));
            if (!plan) throw Fail{GF2E_ERR_CUDA};
            const u64 n = gf2e::fft_plan_n(plan);
            Buf F2[4], F1[4];
            for (int i = 0; i < 4; i++) {
                F2[i] = alloc(G_ * n);
                fwd(plan, M2.e[i], F2[i]->p, n);
                F1[i] = alloc(G_ * n);
                fwd(plan, M1.e[i], F1[i]->p, n);
            }
            Buf O = alloc(G_ * n);
            for (int i = 0; i < 2; i++)
                for (int j = 0; j < 2; j++)
                    r.e[2 * i + j] = product_out(plan, O->p, F2[2 * i]->p, F1[j]->p, F2[2 * i + 1]->p,
                                                 F1[2 + j]->p, n, need,
                                                 sum_bound(M2.e[2 * i], M1.e[j], M2.e[2 * i + 1], M1.e[2 + j]));
            stats.fft_mul2 += 4;
        } else {
            PairB P[4];
            for (int i = 0; i < 2; i++)
                for (int j = 0; j < 2; j++)
                    P[2 * i + j] = PairB{&M2.e[2 * i], &M1.e[j], &M2.e[2 * i + 1], &M1.e[2 + j]};
            mul2_school(P, 4, r.e);
        }
        return r;
    }

    // rows x ^ (q[g] y << s[g]) for the members in `run`, x for the rest
    BPoly axpy_rows(const BPoly &x, const BPoly &y, const std::vector<u64> &q,
                    const std::vector<long long> &s, const Mask &run) {
        BPoly r;
        r.deg.assign(G_, -1);
        r.win.assign(G_, 0);
        u64 stride = 1;
        for (int g = 0; g < G_; g++) {
            long long d = x.deg[g];
            if (run[g] && q[g] && y.deg[g] >= 0) d = std::max(d, y.deg[g] + (63 - __builtin_clzll(q[g])) + s[g]);
            r.deg[g] = d;
            stride = std::max(stride, r.words(g));
        }
        r.stride = stride;
        r.b = alloc((size_t)G_ * stride);
        AxpyBatch A;
        memset(&A, 0, sizeof A);
        A.out = r.base();
        A.so = stride;
        A.x = x.base();
        A.sx = x.stride;
        A.y = y.base();
        A.sy = y.stride;
        for (int g = 0; g < G_; g++) {
            A.q[g] = run[g] ? q[g] : 0;
            A.s[g] = run[g] ? (u64)s[g] : 0;
            A.nx[g] = (u32)x.words(g);
            A.ny[g] = (u32)y.words(g);
            A.nout[g] = (u32)r.words(g);
        }
        k_axpy_b<<<dim3(std::max(1, gf2e::grid_for(stride, 256) / G_ + 1), G_), 256, 0, st_>>>(A);
        ckc(cudaGetLastError(), "k_axpy_b");
        return r;
    }

    // for the members in act (deg c >= deg d >= 0): (c, d) <- (d, c mod d)
    // and, with M, rows (R0, R1) <- (R1, R0 + q R1); the rest unchanged
    void divstep(BPoly &c, BPoly &d, BMat *M, const Mask &act) {
        Timer tm(stats.us_division);
        stats.divsteps++;
        for (int g = 0; g < G_; g++)
            if (act[g] && d.deg[g] < 0) throw Fail{gf2e::invalid("hgcd: division by zero")};
        if (!c.has_win || !d.has_win) probe({&c, &d}, &act);
        BPoly cc = c;
        BPoly r0a, r0b;
        if (M) { r0a = M->e[0]; r0b = M->e[1]; }
        Mask run(G_, 0);
        for (int g = 0; g < G_; g++) run[g] = act[g] && cc.deg[g] >= d.deg[g];
        bool first = true;
        std::vector<u64> q(G_, 0);
        std::vector<long long> s(G_, 0);
        for (int guard = 0; any_of(run); guard++) {
            if (guard > (1 << 22)) throw Fail{gf2e::invalid("hgcd: division did not converge")};
            for (int g = 0; g < G_; g++) {
                q[g] = 0;
                s[g] = 0;
                if (!run[g]) continue;
                const long long delta = cc.deg[g] - d.deg[g];
                const int nb = (int)std::min<long long>(delta, 63);    // quotient bits - 1
                u64 qq = 0, rr = cc.win[g];
                for (int t = 0; t <= nb; t++)
                    if ((rr >> (63 - t)) & 1) {
                        qq |= 1ull << (nb - t);
                        rr ^= d.win[g] >> t;
                    }
                q[g] = qq;
                s[g] = delta - nb;
            }
            // c ^= (q d) << s (in place after the first step: the result is lower)
            BPoly nc = first ? make(cc.stride, false) : cc;
            nc.deg = cc.deg;
            nc.win = cc.win;
            AxpyBatch A;
            memset(&A, 0, sizeof A);
            A.out = nc.base();
            A.so = nc.stride;
            A.x = cc.base();
            A.sx = cc.stride;
            A.y = d.base();
            A.sy = d.stride;
            for (int g = 0; g < G_; g++) {
                A.q[g] = q[g];
                A.s[g] = (u64)s[g];
                A.nx[g] = (u32)cc.words(g);
                A.ny[g] = (u32)d.words(g);
                A.nout[g] = (u32)cc.words(g);
            }
            k_axpy_b<<<dim3(std::max(1, gf2e::grid_for(nc.stride, 256) / G_ + 1), G_), 256, 0, st_>>>(A);
            ckc(cudaGetLastError(), "k_axpy_b");
            if (M) {
                r0a = axpy_rows(r0a, M->e[2], q, s, run);
                r0b = axpy_rows(r0b, M->e[3], q, s, run);
            }
            first = false;
            cc = nc;
            probe({&cc}, &run);
            for (int g = 0; g < G_; g++) run[g] = run[g] && cc.deg[g] >= d.deg[g];
        }
        cc.has_win = false;
        if (all_of(act)) {
            if (M) {
                BPoly n0 = M->e[2], n1 = M->e[3];
                M->e[0] = n0; M->e[1] = n1;
                M->e[2] = r0a; M->e[3] = r0b;
            }
            c = d;
            d = cc;
        } else {
            if (M) {
                BPoly e0 = select(act, M->e[2], M->e[0]), e1 = select(act, M->e[3], M->e[1]);
                BPoly e2 = select(act, r0a, M->e[2]), e3 = select(act, r0b, M->e[3]);
                M->e[0] = e0; M->e[1] = e1; M->e[2] = e2; M->e[3] = e3;
            }
            BPoly nc = select(act, d, c), nd = select(act, cc, d);
            c = nc;
            d = nd;
        }
        c.has_win = false;
        d.has_win = false;
    }

    BMat base(const BPoly &a, const BPoly &b, const std::vector<long long> &m, const Mask &act) {
        Timer tm(stats.us_base);
        stats.bases++;
        long long dmax = 0, emax = 0;
        for (int g = 0; g < G_; g++)
            if (act[g]) {
                dmax = std::max(dmax, a.deg[g]);
                emax = std::max(emax, a.deg[g] - m[g]);
            }
        const u64 W = (u64)(dmax >> 6) + 2;
        const u64 mw = (u64)(emax >> 6) + 3;
        const size_t smem = (4 * W + 8 * mw) * 8;
        if (smem > 200 * 1024) throw Fail{gf2e::invalid("hgcd: base case too large")};
        Buf out = alloc((size_t)G_ * 4 * mw);
        base_smem_attr();
        BaseBatch BB;
        memset(&BB, 0, sizeof BB);
        BB.a = a.base();
        BB.b = b.base();
        BB.sa = a.stride;
        BB.sb = b.stride;
        BB.M = out->p;
        for (int g = 0; g < G_; g++) {
            BB.da[g] = act[g] ? a.deg[g] : 0;
            BB.db[g] = act[g] ? b.deg[g] : -1;
            BB.m[g] = act[g] ? m[g] : 0;
        }
        k_hgcd_base<<<G_, BASE_THREADS, smem, st_>>>(BB, W, mw, (BaseAcc *)d_res_->p);
        ckc(cudaGetLastError(), "k_hgcd_base");
        BMat M;
        for (int i = 0; i < 4; i++) {
            M.e[i].b = view_of(out, (size_t)i * mw, (size_t)(G_ - 1) * 4 * mw + mw);
            M.e[i].stride = 4 * mw;
            M.e[i].win.assign(G_, 0);
            M.e[i].deg.assign(G_, -1);
            for (int g = 0; g < G_; g++)
                M.e[i].deg[g] = act[g] ? std::max(0LL, a.deg[g] - m[g]) : (i == 0 || i == 3 ? 0 : -1);
        }
        return M;
    }

    // deg a > deg b for the members in act_in; exact degrees on entry
    BMat hgcd(const BPoly &a, const BPoly &b, const Mask &act_in) {
        stats.nodes++;
        Mask act(G_, 0);
        std::vector<long long> m(G_, 0);
        long long nmax = -1;
        for (int g = 0; g < G_; g++) {
            m[g] = a.deg[g] < 0 ? 0 : (a.deg[g] + 1) / 2;
            act[g] = act_in[g] && b.deg[g] >= 0 && b.deg[g] >= m[g];
            if (act[g]) nmax = std::max(nmax, a.deg[g]);
        }
        if (!any_of(act)) return identity();
        if (nmax <= tn_.base_bits) return base(a, b, m, act);
        BPoly a1 = shr(a, m, act), b1 = shr(b, m, act);
        BMat M1 = hgcd(a1, b1, act);
        BPoly c, d;
        mat_vec(M1, a, b, c, d);
        Mask sw(G_, 0);
        for (int g = 0; g < G_; g++) sw[g] = act[g] && c.deg[g] < d.deg[g];    // not expected
        if (any_of(sw)) {
            swap_members(sw, c, d);
            M1 = materialize(M1);
            BPoly e0 = select(sw, M1.e[2], M1.e[0]), e1 = select(sw, M1.e[3], M1.e[1]);
            BPoly e2 = select(sw, M1.e[0], M1.e[2]), e3 = select(sw, M1.e[1], M1.e[3]);
            M1.e[0] = e0; M1.e[1] = e1; M1.e[2] = e2; M1.e[3] = e3;
        }
        Mask act2(G_, 0);
        for (int g = 0; g < G_; g++) act2[g] = act[g] && d.deg[g] >= m[g];
        if (!any_of(act2)) return M1;
        M1 = materialize(M1);
        divstep(c, d, &M1, act2);
        Mask act3(G_, 0);
        std::vector<long long> k(G_, 0);
        for (int g = 0; g < G_; g++) {
            act3[g] = act2[g] && d.deg[g] >= m[g];
            if (act3[g]) k[g] = std::max(0LL, 2 * m[g] - c.deg[g]);
        }
        if (!any_of(act3)) return M1;
        BPoly c1 = shr(c, k, act3), d1 = shr(d, k, act3);
        BMat M2 = hgcd(c1, d1, act3);
        return mat_mul(M2, M1);
    }

    // the quadratic gcd (gcd.cu) for the members in fin, one batch
    void small_gcds(const BPoly &a, const BPoly &b, const Mask &fin, BPoly &sg,
                    std::vector<Buf> &keep, std::vector<u64 *> &ptr) {
        Timer tm(stats.us_small);
        std::vector<gf2e_gcd_job> J;
        std::vector<int> who;
        for (int g = 0; g < G_; g++) {
            if (!fin[g]) continue;
            gf2e_gcd_job job;
            memset(&job, 0, sizeof job);
            job.a_dev = a.base() + (u64)g * a.stride;
            job.abits = (u64)a.deg[g] + 1;
            job.b_dev = b.base() + (u64)g * b.stride;
            job.bbits = (u64)b.deg[g] + 1;
            const u64 gw = (u64)(std::max(a.deg[g], b.deg[g]) >> 6) + 2;
            Buf out = alloc(gw);
            ckc(cudaMemsetAsync(out->p, 0, gw * 8, st_), "hgcd memset");
            job.g_dev = out->p;
            job.g_cap_words = gw;
            keep.push_back(out);
            ptr[g] = out->p;
            J.push_back(job);
            who.push_back(g);
        }
        size_t need = 0;
        ck(gf2e_gcd_workspace_size(J.data(), (int)J.size(), &need));
        Buf ws = alloc((need + 7) / 8);
        std::vector<int64_t> degs(J.size(), -1);
        ck(gf2e_gcd_batch(J.data(), (int)J.size(), degs.data(), ws->p, need, st_));
        for (size_t i = 0; i < who.size(); i++) sg.deg[who[i]] = degs[i];
    }

    void finish_bases() {
        BaseAcc acc;
        ckc(cudaMemcpyAsync(&acc, d_res_->p, sizeof acc, cudaMemcpyDeviceToHost, st_), "base totals");
        ckc(cudaStreamSynchronize(st_), "base totals sync");
        stats.base_rounds = (long long)acc.rounds;
        stats.cyc_serial = (long long)acc.cyc_serial;
        stats.cyc_total = (long long)acc.cyc_total;
        if (acc.worst != GF2E_OK) {
            gf2e::set_error("hgcd base case status %d", acc.worst);
            throw Fail{acc.worst};
        }
    }

    Arena arena_;                      // declared first: destroyed after every buffer
    int G_;
    cudaStream_t st_;
    Tunables tn_;
    long long *h_probe_ = nullptr;
    Buf d_probe_, d_res_;
};

cudaMemPool_t hgcd_pool() {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 0 || dev >= 64) return nullptr;
    if (!pools[dev]) {
        cudaMemPoolProps props;
        memset(&props, 0, sizeof props);
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        if (cudaMemPoolCreate(&pools[dev], &props) != cudaSuccess) return nullptr;
        u64 keep = ~0ull;      // keep freed memory in the pool between gcds
        cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
    }
    return pools[dev];
}

// members in flight: the caller's cap, GMAX, and what device memory holds
// (per member about 40 operand-sized buffers and 12 transforms of the
// largest matrix product: 1.52 GB measured at r = 136279841), counting as
// free what the gcd pool holds from earlier gcds but does not use
int batch_size(cudaMemPool_t pool, const gf2e_gcd_job *jobs, int njobs, int max_parallel) {
    u64 bits = 1;
    for (int i = 0; i < njobs; i++) bits = std::max(bits, std::max(jobs[i].abits, jobs[i].bbits));
    const u64 words = (bits + 63) / 64;
    u64 n = 1;
    while (n < (3 * bits / 2) / 32 + 1) n <<= 1;
    const double per = 8.0 * (40.0 * (double)words + 12.0 * (double)n);
    size_t fr = 0, tot = 0;
    int cap = GMAX;
    if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) {
        unsigned long long reserved = 0, used = 0;
        if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
            cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess &&
            reserved > used)
            fr += (size_t)(reserved - used);
        cap = (int)std::max(1.0, std::min((double)GMAX, 0.9 * (double)fr / per));
    }
    return std::max(1, std::min(std::min(njobs, max_parallel), cap));
}

void add_stats(gf2e_hgcd_stats &t, const Stats &s) {
    t.nodes += s.nodes;
    t.base_cases += s.bases;
    t.base_rounds += s.base_rounds;
    t.fft_products += s.fft_mul2;
    t.school_products += s.school_mul2;
    t.division_steps += s.divsteps;
    t.probes += s.probes;
    t.us_base += (int64_t)s.us_base;
    t.us_products += (int64_t)s.us_products;
    t.us_division += (int64_t)s.us_division;
    t.us_small_gcd += (int64_t)s.us_small;
    t.base_cycles_serial += s.cyc_serial;
    t.base_cycles_total += s.cyc_total;
}

// lockstep batches: the members in flight (the memory cap) split over
// `streams` batches that run at once, each on its own host thread and
// stream, so that one batch's base cases (a CTA per member, most SMs idle)
// overlap another's products; further batches follow as these finish
int run_lockstep(const gf2e_gcd_job *jobs, int njobs, int64_t *deg_host, int max_parallel,
                 gf2e_hgcd_stats *stats) {
    cudaMemPool_t pool = hgcd_pool();
    if (!pool) return gf2e::cuda_status(cudaErrorMemoryAllocation, "hgcd memory pool");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return gf2e::cuda_status(e, "hgcd device");
    if (stats) memset(stats, 0, sizeof *stats);
    const int B = batch_size(pool, jobs, njobs, max_parallel);
    const int lanes = std::max(1, std::min(tunables(true).streams, B / 8));
    const int per = (B + lanes - 1) / lanes;
    std::atomic<int> next(0);
    std::mutex mu;
    int rc = GF2E_OK;
    auto worker = [&]() {
        cudaSetDevice(dev);
        cudaStream_t st;
        cudaError_t ce = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        if (ce != cudaSuccess) {
            std::lock_guard<std::mutex> lk(mu);
            rc = gf2e::cuda_status(ce, "hgcd stream");
            return;
        }
        // a batch that runs out of device memory (the other batch in flight,
        // or the estimate) is retried as two halves
        auto run_members = [&](auto &&self, int i0, int nb) -> int {
            try {
                HgcdBatch H(nb, st, pool);
                H.run(jobs + i0, deg_host + i0);
                std::lock_guard<std::mutex> lk(mu);
                if (stats) add_stats(*stats, H.stats);
                return GF2E_OK;
            } catch (const Fail &f) {
                cudaStreamSynchronize(st);
                if (f.st != GF2E_ERR_NOMEM || nb == 1) return f.st;
            } catch (const std::exception &x) {        // host allocation and the like
                cudaStreamSynchronize(st);
                gf2e::set_error("hgcd: %s", x.what());
                return GF2E_ERR_INTERNAL;
            }
            const int h = nb / 2;
            const int r1 = self(self, i0, h);
            return r1 != GF2E_OK ? r1 : self(self, i0 + h, nb - h);
        };
        for (int b; (b = next.fetch_add(1)) * per < njobs;) {
            const int i0 = b * per;
            const int r1 = run_members(run_members, i0, std::min(per, njobs - i0));
            if (r1 != GF2E_OK) {
                std::lock_guard<std::mutex> lk(mu);
                if (rc == GF2E_OK) rc = r1;
            }
        }
        cudaStreamDestroy(st);
    };
    if (lanes == 1) {
        worker();
    } else {
        std::vector<std::thread> th;
        for (int t = 0; t < lanes; t++) th.emplace_back(worker);
        for (auto &t : th) t.join();
    }
    return rc;
}

}  // namespace

extern "C" {

int gf2e_gcd_large(const gf2e_gcd_job *jobs, int njobs, int64_t *deg_host, int max_parallel,
                   gf2e_hgcd_stats *stats, void *stream) {
    if (!jobs || njobs < 1 || !deg_host) return gf2e::invalid("gf2e_gcd_large: bad job list");
    for (int i = 0; i < njobs; i++)
        if (!jobs[i].a_dev || !jobs[i].b_dev || !jobs[i].abits || !jobs[i].bbits)
            return gf2e::invalid("gf2e_gcd_large: empty operand in job %d", i);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return gf2e::cuda_status(e, "gf2e_gcd_large device");
    // the caller's stream must have produced the operands before we start
    cudaEvent_t ready;
    e = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(ready, (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(ready);
    cudaEventDestroy(ready);
    if (e != cudaSuccess) return gf2e::cuda_status(e, "gf2e_gcd_large operands");
    return run_lockstep(jobs, njobs, deg_host, std::max(1, max_parallel), stats);
}

}  // extern "C"
