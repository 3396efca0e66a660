// cantor.cu -- Cantor additive FFT over GF(2^64) and GF(2)[x] multiply.
//
// Transform definition (points, order, twiddles) is the reference's
// (gf2_cantor_engine.h:125-188): a Taylor cascade of range-XORs for depths
// L = 0..m-2, then butterflies for levels m-1..0 with twiddle
// W[t] = XOR of basis[j+1] over the set bits j of t.
//
// B200 mapping.  Every Taylor level and butterfly level acts on "rows" of a
// strided 2-D view of the array, so a run of consecutive levels fits in one
// shared-memory tile of NS rows (row stride CH elements) x C contiguous
// columns.  One kernel launch (a "pass") loads each tile once from HBM,
// applies up to ~10 levels in shared memory and stores it once.  Once the
// depth L0 is reached at which a whole depth-L0 subproblem (n >> L0 rows of
// the view) fits in a tile, one pass finishes every remaining Taylor depth
// and the matching butterfly levels (m-1..L0) for a group of columns.  At
// m = 24 with 4096-element tiles this is ~36 passes per transform instead of
// the reference's ~70 fused / ~550 legacy passes.  Twiddles are rebuilt
// from four 256-entry byte tables (W is GF(2)-linear in t), so no n/2-entry
// table is streamed from HBM.
#include "gf2e_internal.cuh"
#include "wrapmul.cuh"

#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>
#include <algorithm>
#include <atomic>

namespace {

// shared-memory tiles are 2^11..2^13 elements (16..64 KB), chosen per plan
constexpr int MAXOPS = 96;
constexpr int FFT_THREADS = 512;           // one CTA per SM, double-buffered tiles
constexpr int NTWTAB = 4;                  // byte tables: t < 2^32

enum OpType : u32 { TAY_F = 0, TAY_I = 1, BF_F = 2, BF_I = 3 };

// op word: type | log2(row quarter or row distance) << 2 | L << 8
__host__ __device__ inline u32 mkop(u32 type, u32 lg, u32 L) { return type | (lg << 2) | (L << 8); }

struct Pass {
    u64 CH;          // row stride (elements)
    u32 ns_log;      // log2 rows per window
    u32 c_log;       // log2 columns per tile
    u32 wpt_log;     // log2 windows per tile (only when C == CH)
    u32 nops;
    u32 ops[MAXOPS];
    u32 stream;      // 1: a streaming Taylor level over HBM (no tile), below
    u32 sM, sA;      // its block 2^sM and chunk 2^sA elements
};

// A Taylor level at x^tau + x, tau = 2^(M-1-a), on aligned blocks of 2^M
// elements in chunks of c = 2^a.  With the Cantor basis x^(2^h) + x is the
// subspace polynomial of degree 2^h whenever h is a power of two, so the
// conversion of 2^m coefficients to the products-of-subspace-polynomials
// basis (what the reference's cascade of x^2 + x levels computes) splits
// into m - h levels at tau = 2^h (h the largest power of two below m) and
// two independent conversions of 2^h and 2^(m-h) coefficients (Gao and
// Mateer's recursion): at m = 24, 16 streamed tau levels and three 8-bit
// cascades (84 levels in 3 tile passes) instead of 276 cascade levels.
//   forward: Hi[0..c) ^= Top; A[c..B) ^= Hi[0..B-c)   (B = 2^(M-1), A = the
//            first half, Hi the second, Top its last c elements)
//   inverse: A[c..B) ^= Hi[0..B-c); Hi[0..c) ^= Top
// tau = 2 is the cascade's level (TAY_F / TAY_I ops in tile passes).

// W(t) from byte tables: tab[k*256 + b] = XOR of basis[8k+j+1], bits j of b
GF2E_DEV u64 twiddle(const u64 *__restrict__ tab, u64 t) {
    u64 w = 0;
#pragma unroll
    for (int k = 0; k < NTWTAB; k++) w ^= __ldg(tab + k * 256 + ((t >> (8 * k)) & 255));
    return w;
}

// Tile rows are XOR-swizzled in shared memory so that the rows a warp
// touches at power-of-two distances fall in different banks.  The swizzle
// only permutes rows inside aligned groups of 16, so it is a bijection on
// any power-of-two row count.
GF2E_DEV u32 srow(u32 row) { return row ^ (((row >> 4) ^ (row >> 8) ^ (row >> 12)) & 15); }
GF2E_DEV u32 sidx(u32 row, u32 col, u32 c_log) { return (srow(row) << c_log) + col; }

// A stage applies K consecutive Taylor levels in registers.  Row quarters
// q*2^(K-1) .. q (q = 2^lg rows): each thread holds the 2^(K+1) rows
// row0 + j*q of one column, with row0 = blk * q * 2^(K+1) + i, i < q.
// Forward goes from the largest blocks down, inverse the other way.
//
// Shared-memory indices: row0 has no bits in [lg, lg+K+1) and the swizzle is
// linear over XOR, so the index of row row0 + j*q is the group's base index
// XOR off[j] = srow(j << lg) << c_log, a per-stage table built once per CTA.
template <bool FWD, int K>
GF2E_DEV void taylor_stage(u64 *sm, const u32 *off, u32 lg, u32 c_log, u32 tile_elems) {
    constexpr int R = 2 << K;                       // rows per thread
    const u32 C = 1u << c_log, q = 1u << lg;
    const u32 ngroups = tile_elems / R;
    for (u32 g = threadIdx.x; g < ngroups; g += FFT_THREADS) {
        const u32 col = g & (C - 1), rest = g >> c_log;
        const u32 i = rest & (q - 1), blk = rest >> lg;
        const u32 row0 = (blk << (lg + K + 1)) + i;
        const u32 b0 = (srow(row0) << c_log) | col;
        u64 v[R];
#pragma unroll
        for (int j = 0; j < R; j++) v[j] = sm[b0 ^ off[j]];
        if (FWD) {
#pragma unroll
            for (int lev = K - 1; lev >= 0; lev--) {
                const int Q = 1 << lev;
#pragma unroll
                for (int o = 0; o < R; o += 4 * Q)
#pragma unroll
                    for (int ii = 0; ii < Q; ii++) {
                        v[o + 2 * Q + ii] ^= v[o + 3 * Q + ii];
                        v[o + Q + ii] ^= v[o + 2 * Q + ii];
                    }
            }
        } else {
#pragma unroll
            for (int lev = 0; lev < K; lev++) {
                const int Q = 1 << lev;
#pragma unroll
                for (int o = 0; o < R; o += 4 * Q)
#pragma unroll
                    for (int ii = 0; ii < Q; ii++) {
                        v[o + Q + ii] ^= v[o + 2 * Q + ii];
                        v[o + 2 * Q + ii] ^= v[o + 3 * Q + ii];
                    }
            }
        }
#pragma unroll
        for (int j = 0; j < R; j++) sm[b0 ^ off[j]] = v[j];
    }
}

// A stage of K consecutive butterfly levels in registers: row distances
// D*2^(K-1) .. D (D = 2^lg rows, physical level Llo for distance D).  A
// thread holds the 2^K rows row0 + j*D of one column.  The twiddle of the
// pair at j in level Llo+lev is W[(Q0 + j) >> (lev+1)], Q0 = (base >> Llo) +
// blk*2^K; Q0 is a multiple of 2^K, so by linearity of W it is
// W[Q0 >> (lev+1)] ^ W[j >> (lev+1)], the second term from the first byte
// table (j < 8).
template <bool FWD, int K>
GF2E_DEV void bfly_stage(u64 *sm, const u32 *off, const u64 *__restrict__ tab, u32 lg, u32 Llo,
                         u32 c_log, u32 tile_elems, u64 base) {
    constexpr int R = 1 << K;
    const u32 C = 1u << c_log, D = 1u << lg;
    const u32 ngroups = tile_elems / R;
    for (u32 g = threadIdx.x; g < ngroups; g += FFT_THREADS) {
        const u32 col = g & (C - 1), rest = g >> c_log;
        const u32 i = rest & (D - 1), blk = rest >> lg;
        const u32 row0 = (blk << (lg + K)) + i;
        const u32 b0 = (srow(row0) << c_log) | col;
        const u64 Q0 = (base >> Llo) + ((u64)blk << K);
        u64 v[R];
#pragma unroll
        for (int j = 0; j < R; j++) v[j] = sm[b0 ^ off[j]];
#pragma unroll
        for (int step = 0; step < K; step++) {
            const int lev = FWD ? K - 1 - step : step;
            const int Dj = 1 << lev;
            const u64 tb = twiddle(tab, Q0 >> (lev + 1));
#pragma unroll
            for (int j = 0; j < R; j++) {
                if (j & Dj) continue;
                const u64 tw = tb ^ ((j >> (lev + 1)) ? __ldg(tab + (j >> (lev + 1))) : 0ull);
                if (FWD) {
                    // W[0] = 0: the first block of every level multiplies by
                    // zero (all of level m-1, half of m-2, ...), warp-uniformly
                    u64 e = v[j] ^ (tw ? gf64_mul(tw, v[j + Dj]) : 0ull);
                    v[j + Dj] ^= e;
                    v[j] = e;
                } else {
                    u64 hh = v[j] ^ v[j + Dj];
                    if (tw) v[j] ^= gf64_mul(tw, hh);
                    v[j + Dj] = hh;
                }
            }
        }
#pragma unroll
        for (int j = 0; j < R; j++) sm[b0 ^ off[j]] = v[j];
    }
}

// Batch description for one pass: blockIdx.y selects the transform
// (f + y*fstride) and its operand (src32 + y*sstride32).  xor0 is XORed into
// chunk 0 of every packed operand (the running product multiplies by F + x).
struct Batch {
    u64 fstride;
    u64 sstride32;
    u64 xor0;
};

// One pass over all tiles.  src32/nchunks: when non-null the tile is loaded
// from 32-bit chunks of an operand (packing fused into the first pass),
// zero beyond nchunks.
// asynchronous 8-byte global -> shared copies (completion by group)
GF2E_DEV void cp_async8(u64 *smem_dst, const u64 *gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
GF2E_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
GF2E_DEV void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// One pass over all tiles.  src32/nchunks: when non-null the tile is loaded
// from 32-bit chunks of an operand (packing fused into the first pass),
// zero beyond nchunks.
//
// DB (large passes): each CTA runs over its tiles with two tile buffers in
// shared memory, the next tile fetched with asynchronous copies while the
// current one is transformed and stored, so HBM traffic overlaps the stage
// work (the packing pass, which converts 32-bit chunks, loads
// synchronously).  Without DB (passes with few tiles per CTA) one buffer,
// synchronous loads and two CTAs per SM.
template <int TL, bool DB>
__global__ void __launch_bounds__(FFT_THREADS, DB ? 1 : 2)
k_fft_pass(u64 *__restrict__ f, const u64 *__restrict__ tab, const Pass P, u64 ntiles,
           const u32 *__restrict__ src32, u64 nchunks, const Batch bt) {
    extern __shared__ u64 smbuf[];                   // one or two tiles of 2^TL elements
    __shared__ u32 s_off[MAXOPS * 16];               // per stage: srow(j << lg) << c_log
    __shared__ u32 s_loff[16];                       // load/store rows: srow(j << rs) << c_log
    f += (u64)blockIdx.y * bt.fstride;
    if (src32) src32 += (u64)blockIdx.y * bt.sstride32;
    const u32 C = 1u << P.c_log;
    const u32 NS = 1u << P.ns_log;
    const u32 rows_total = NS << P.wpt_log;          // rows in the tile (all windows)
    const u32 tile_elems = rows_total * C;
    const u64 cgroups = P.CH >> P.c_log;             // column groups per window
    // element e = tid + j*FFT_THREADS of the tile is (row_t + j << rs, col_t)
    // when a row holds at most FFT_THREADS columns; its swizzled index is the
    // thread's base index XOR s_loff[j] (rows and the swizzle are linear)
    constexpr u32 THREADS_LOG = 9;
    static_assert((1 << THREADS_LOG) == FFT_THREADS, "thread count");
    const bool fast = P.c_log <= THREADS_LOG;
    const u32 rs = fast ? THREADS_LOG - P.c_log : 0;
    const u32 row_t = threadIdx.x >> P.c_log, col_t = threadIdx.x & (C - 1);
    const u32 sb_t = (srow(row_t) << P.c_log) | col_t;
    for (u32 t = threadIdx.x; t < P.nops * 16; t += FFT_THREADS) {
        const u32 lg = (P.ops[t >> 4] >> 2) & 63;
        s_off[t] = srow((t & 15) << lg) << P.c_log;
    }
    if (threadIdx.x < 16) s_loff[threadIdx.x] = srow(threadIdx.x << rs) << P.c_log;
    __syncthreads();
    constexpr int EPT = (1 << TL) / FFT_THREADS;
    const u64 g_step = P.CH << rs;

    auto tile_base = [&](u64 tile) -> u64 {
        if (P.wpt_log) return tile * ((u64)tile_elems);       // several whole windows, C == CH
        const u64 win = tile / cgroups, cg = tile - win * cgroups;
        return win * ((u64)NS * P.CH) + cg * C;
    };
    // issue the loads of `tile` into buffer `sm` (asynchronous unless packing)
    auto load_tile = [&](u64 tile, u64 *sm) {
        const u64 base = tile_base(tile);
        const u64 g_t = base + (u64)row_t * P.CH + col_t;
        if (src32 || !DB) {
#pragma unroll
            for (int j0 = 0; j0 < EPT; j0 += 8) {
                u64 v[8];
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const u32 e = threadIdx.x + (j0 + j) * FFT_THREADS;
                    v[j] = 0;
                    if (j0 + j < EPT && e < tile_elems) {
                        const u64 g = fast ? g_t + (u64)(j0 + j) * g_step
                                           : base + (u64)(e >> P.c_log) * P.CH + (e & (C - 1));
                        if (src32) {
                            v[j] = (g < nchunks) ? (u64)__ldg(src32 + g) : 0ull;
                            if (g == 0) v[j] ^= bt.xor0;
                        } else {
                            v[j] = f[g];
                        }
                    }
                }
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const u32 e = threadIdx.x + (j0 + j) * FFT_THREADS;
                    if (j0 + j < EPT && e < tile_elems)
                        sm[fast ? (sb_t ^ s_loff[j0 + j]) : sidx(e >> P.c_log, e & (C - 1), P.c_log)] = v[j];
                }
            }
        } else {
#pragma unroll
            for (int j = 0; j < EPT; j++) {
                const u32 e = threadIdx.x + j * FFT_THREADS;
                if (e < tile_elems) {
                    if (fast) cp_async8(sm + (sb_t ^ s_loff[j]), f + g_t + (u64)j * g_step);
                    else cp_async8(sm + sidx(e >> P.c_log, e & (C - 1), P.c_log),
                                   f + base + (u64)(e >> P.c_log) * P.CH + (e & (C - 1)));
                }
            }
        }
        if (DB) cp_async_commit();
    };

    u64 tile = blockIdx.x;
    if (DB) {
        if (tile < ntiles) load_tile(tile, smbuf);
        else cp_async_commit();
    }
    for (int it = 0; tile < ntiles; tile += gridDim.x, it++) {
        u64 *sm = DB ? smbuf + ((it & 1) << TL) : smbuf;
        if (DB) {
            const u64 next = tile + gridDim.x;
            if (next < ntiles) load_tile(next, smbuf + (((it + 1) & 1) << TL));
            else cp_async_commit();                    // keep one group per iteration
            cp_async_wait_prev();                      // this tile's copies are done
        } else {
            load_tile(tile, sm);
        }
        __syncthreads();
        const u64 base = tile_base(tile);
        for (u32 k = 0; k < P.nops; k++) {
            const u32 op = P.ops[k];
            const u32 type = op & 3, lg = (op >> 2) & 63, L = (op >> 8) & 127;
            const u32 K = ((op >> 15) & 3) + 1;
            const u32 *off = s_off + k * 16;
            switch (type * 4 + K) {
            case TAY_F * 4 + 1: taylor_stage<true, 1>(sm, off, lg, P.c_log, tile_elems); break;
            case TAY_F * 4 + 2: taylor_stage<true, 2>(sm, off, lg, P.c_log, tile_elems); break;
            case TAY_F * 4 + 3: taylor_stage<true, 3>(sm, off, lg, P.c_log, tile_elems); break;
            case TAY_I * 4 + 1: taylor_stage<false, 1>(sm, off, lg, P.c_log, tile_elems); break;
            case TAY_I * 4 + 2: taylor_stage<false, 2>(sm, off, lg, P.c_log, tile_elems); break;
            case TAY_I * 4 + 3: taylor_stage<false, 3>(sm, off, lg, P.c_log, tile_elems); break;
            case BF_F * 4 + 1: bfly_stage<true, 1>(sm, off, tab, lg, L, P.c_log, tile_elems, base); break;
            case BF_F * 4 + 2: bfly_stage<true, 2>(sm, off, tab, lg, L, P.c_log, tile_elems, base); break;
            case BF_F * 4 + 3: bfly_stage<true, 3>(sm, off, tab, lg, L, P.c_log, tile_elems, base); break;
            case BF_I * 4 + 1: bfly_stage<false, 1>(sm, off, tab, lg, L, P.c_log, tile_elems, base); break;
            case BF_I * 4 + 2: bfly_stage<false, 2>(sm, off, tab, lg, L, P.c_log, tile_elems, base); break;
            case BF_I * 4 + 3: bfly_stage<false, 3>(sm, off, tab, lg, L, P.c_log, tile_elems, base); break;
            default: break;                    // butterfly stages hold at most 3 levels
            }
            __syncthreads();
        }
        if (fast) {
            const u64 g_t = base + (u64)row_t * P.CH + col_t;
#pragma unroll
            for (int j = 0; j < EPT; j++) {
                const u32 e = threadIdx.x + j * FFT_THREADS;
                if (e < tile_elems) f[g_t + (u64)j * g_step] = sm[sb_t ^ s_loff[j]];
            }
        } else {
            for (u32 e = threadIdx.x; e < tile_elems; e += FFT_THREADS) {
                u32 row = e >> P.c_log, col = e & (C - 1);
                f[base + (u64)row * P.CH + col] = sm[sidx(row, col, P.c_log)];
            }
        }
        __syncthreads();                               // buffer free for the load after next
    }
    if (DB) asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// one tau level streamed over HBM for levels whose blocks span more rows
// than a tile holds (tau >= 2^10); V elements per item (16-byte accesses
// when chunks are at least 2 elements).  blockIdx.y selects the transform.
template <int V>
__global__ void k_tau_stream(u64 *__restrict__ f, u64 fstride, u64 n, int M, int a, int fwd) {
    f += (u64)blockIdx.y * fstride;
    const u64 half = 1ull << (M - 1), c = 1ull << a, nq = half - c;
    const u64 items = (n >> 1) / V;
    for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < items;
         t += (u64)gridDim.x * blockDim.x) {
        const u64 e = t * V, blk = e >> (M - 1), q = e & (half - 1);
        if (q >= nq) continue;
        const u64 b0 = blk << M;
        u64 *A = f + b0 + c + q, *H = f + b0 + half + q;
        const u64 *T = f + b0 + 2 * half - c + q;
        if (V == 2) {
            ulonglong2 h = *reinterpret_cast<const ulonglong2 *>(H);
            ulonglong2 x = *reinterpret_cast<const ulonglong2 *>(A);
            if (fwd) {
                if (q < c) {
                    const ulonglong2 tp = *reinterpret_cast<const ulonglong2 *>(T);
                    h.x ^= tp.x;
                    h.y ^= tp.y;
                    *reinterpret_cast<ulonglong2 *>(H) = h;
                }
                x.x ^= h.x;
                x.y ^= h.y;
            } else {
                x.x ^= h.x;
                x.y ^= h.y;
                if (q < c) {
                    const ulonglong2 tp = *reinterpret_cast<const ulonglong2 *>(T);
                    *reinterpret_cast<ulonglong2 *>(H) = make_ulonglong2(h.x ^ tp.x, h.y ^ tp.y);
                }
            }
            *reinterpret_cast<ulonglong2 *>(A) = x;
        } else {
            u64 h = *H;
            if (fwd) {
                if (q < c) { h ^= *T; *H = h; }
                *A ^= h;
            } else {
                *A ^= h;
                if (q < c) *H = h ^ *T;
            }
        }
    }
}

// 32-bit chunks of each operand into the low halves of its transform buffer
// (zero beyond nchunks, xor0 into chunk 0), for transforms whose first pass
// streams instead of loading tiles
__global__ void k_pack_batch(const u32 *__restrict__ src32, u64 sstride32, u64 nchunks, u64 xor0,
                             u64 *__restrict__ f, u64 fstride, u64 n) {
    f += (u64)blockIdx.y * fstride;
    src32 += (u64)blockIdx.y * sstride32;
    for (u64 k = (u64)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (u64)gridDim.x * blockDim.x) {
        u64 v = k < nchunks ? (u64)__ldg(src32 + k) : 0ull;
        if (k == 0) v ^= xor0;
        f[k] = v;
    }
}

__global__ void k_pointwise(u64 *__restrict__ fa, const u64 *__restrict__ fb, u64 n) {
    for (u64 k = (u64)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (u64)gridDim.x * blockDim.x)
        fa[k] = gf64_mul(fa[k], fb[k]);
}

// gather-form overlap-add of 64-bit coefficients at 32-bit stride;
// blockIdx.y selects F + y*fstride -> out + y*ostride
__global__ void k_overlap_add(const u64 *__restrict__ F, u64 nchunks, u64 *__restrict__ out,
                              u64 ow, u64 fstride = 0, u64 ostride = 0) {
    F += (u64)blockIdx.y * fstride;
    out += (u64)blockIdx.y * ostride;
    for (u64 w = (u64)blockIdx.x * blockDim.x + threadIdx.x; w < ow;
         w += (u64)gridDim.x * blockDim.x) {
        u64 k = 2 * w, v = 0;
        if (k < nchunks) v ^= F[k];
        if (k + 1 < nchunks) v ^= F[k + 1] << 32;
        if (w && k - 1 < nchunks) v ^= F[k - 1] >> 32;
        out[w] = v;
    }
}

// ------------------------------------------------------------- host side
u64 host_gf64_mul(u64 a, u64 b) {
    u64 lo = 0, hi = 0;
    for (int i = 0; i < 64; i++)
        if ((b >> i) & 1) {
            lo ^= a << i;
            if (i) hi ^= a >> (64 - i);
        }
    u64 t = lo ^ hi ^ (hi << 1) ^ (hi << 3) ^ (hi << 4);
    u64 h2 = (hi >> 63) ^ (hi >> 61) ^ (hi >> 60);
    return t ^ h2 ^ (h2 << 1) ^ (h2 << 3) ^ (h2 << 4);
}

// Cantor basis: b0 = 1, b_i^2 + b_i = b_{i-1}; of the two solutions
// {y, y+1} the one with zero constant coefficient is taken (the choice the
// reference's elimination makes, gf2_cantor_engine.h:78-103).
int host_cantor_basis(u64 *b) {
    u64 pv[64] = {0}, pt[64] = {0};
    for (int i = 1; i < 64; i++) {
        u64 e = 1ull << i, v = host_gf64_mul(e, e) ^ e, t = e;
        for (int bit = 63; bit >= 0 && v; bit--) {
            if (!((v >> bit) & 1)) continue;
            if (pv[bit]) { v ^= pv[bit]; t ^= pt[bit]; }
            else { pv[bit] = v; pt[bit] = t; v = 0; }
        }
    }
    b[0] = 1;
    int len = 1;
    while (len < 64) {
        u64 c = b[len - 1], v = c, y = 0;
        bool ok = true;
        for (int bit = 63; bit >= 0 && v; bit--) {
            if (!((v >> bit) & 1)) continue;
            if (!pv[bit]) { ok = false; break; }
            v ^= pv[bit];
            y ^= pt[bit];
        }
        if (!ok || v) break;
        y &= ~1ull;
        if ((host_gf64_mul(y, y) ^ y) != c) return -1;
        b[len++] = y;
    }
    return len;
}

const u64 *basis_host() {
    static u64 b[64];
    static int len = 0;
    static std::once_flag once;
    std::call_once(once, [] { len = host_cantor_basis(b); });
    return len == 64 ? b : nullptr;
}

// smallest column count fitting the tile, or 0 if the group does not fit
u32 choose_c(u64 CH, u64 NS, const gf2e_tune &cfg) {
    const u64 tile = (u64)1 << cfg.fft_tile_log;
    if (NS > tile) return 0;
    u64 c = std::min<u64>(CH, tile / NS);
    if (c < (u64)cfg.fft_cmin && c != CH) return 0;
    return (u32)c;
}

int ilog2u(u64 v) { return 63 - __builtin_clzll(v); }

Pass make_pass(u64 CH, u64 NS, u32 C, u64 n, const gf2e_tune &cfg) {
    Pass p;
    memset(&p, 0, sizeof p);
    p.CH = CH;
    p.ns_log = (u32)ilog2u(NS);
    p.c_log = (u32)ilog2u(C);
    // whole windows: pack several into one tile (never more than exist)
    if ((u64)C == CH) {
        u64 win_elems = NS * CH;
        u64 wpt = std::min<u64>(((u64)1 << cfg.fft_tile_log) / win_elems, n / win_elems);
        if (wpt < 1) wpt = 1;
        p.wpt_log = (u32)ilog2u(wpt);
    }
    return p;
}

struct PlanImpl {
    int m = 0;
    u64 n = 0;
    gf2e_tune cfg{};                     // tile size and stage depths the passes use
    u64 *d_tab = nullptr;                // owned NTWTAB x 256 twiddle byte tables
    const u64 *tab = nullptr;            // tables the passes read (d_tab or caller's)
    std::vector<Pass> fwd, inv;
    std::vector<u64> ntiles_fwd, ntiles_inv;
};

// Merge runs of up to three single-level ops of one kind into register
// stages: forward kinds come with the level (lg) falling by one per op,
// inverse kinds with it rising; a stage is encoded by its lowest lg and L
// and its level count K (bits 15-16 hold K-1).
void merge_stages(Pass &p, const gf2e_tune &cfg) {
    u32 out[MAXOPS];
    u32 n = 0;
    for (u32 k = 0; k < p.nops;) {
        const u32 op = p.ops[k], type = op & 3, lg = (op >> 2) & 63, L = (op >> 8) & 127;
        const bool fwd = (type == TAY_F || type == BF_F);
        u32 run = 1;
        const u32 max_run = (u32)((type >= BF_F) ? cfg.fft_bfly_lv : cfg.fft_taylor_lv);
        while (run < max_run && k + run < p.nops) {
            const u32 o2 = p.ops[k + run];
            const u32 lg2 = (o2 >> 2) & 63, L2 = (o2 >> 8) & 127;
            const int want = fwd ? -(int)run : (int)run;
            if ((o2 & 3) != type || (int)lg2 - (int)lg != want) break;
            if (type >= BF_F && (int)L2 - (int)L != want) break;
            run++;
        }
        const u32 lo_lg = fwd ? lg - (run - 1) : lg;
        const u32 lo_L = (type >= BF_F) ? (fwd ? L - (run - 1) : L) : 0;
        out[n++] = mkop(type, lo_lg, lo_L) | ((run - 1) << 15);
        k += run;
    }
    for (u32 k = 0; k < n; k++) p.ops[k] = out[k];
    p.nops = n;
}

u64 pass_tiles(const Pass &p, u64 n) {
    if (p.stream) return 0;
    u64 elems = ((u64)1 << (p.ns_log + p.c_log + p.wpt_log));
    return n / elems;
}

// tau levels (block log M, chunk log a) converting the coefficients whose
// index bits lie in [lo, hi), in an order valid for the forward transform.
// Conversions of at most `cascade_bits` bits use the reference's x^2 + x
// cascade (a = M - 2), whose levels a tile pass applies three at a time in
// registers; wider ones split by Gao and Mateer's recursion into tau levels
// (each streamed over HBM) and two narrower conversions.
void tau_levels(int lo, int hi, int cascade_bits, std::vector<std::pair<int, int>> &out) {
    const int m = hi - lo;
    if (m <= 1) return;
    if (m <= cascade_bits) {
        for (int L = 0; L <= m - 2; L++)
            for (int b = m - L; b >= 2; b--) out.push_back({lo + b + L, lo + b + L - 2});
        return;
    }
    int h = 1;
    while (2 * h < m) h *= 2;
    for (int M = m; M > h; M--) out.push_back({lo + M, lo + M - 1 - h});
    tau_levels(lo + h, hi, cascade_bits, out);    // the 2^(m-h)-coefficient conversions
    tau_levels(lo, lo + h, cascade_bits, out);    // the 2^h-coefficient conversions
}

// the Taylor stage by tau levels (fewer passes) from m = 15 on;
// GF2E_FFT_TAYLOR=cascade keeps the x^2 + x cascade, =tau forces tau levels
bool use_tau_levels(int m) {
    const char *e = getenv("GF2E_FFT_TAYLOR");
    if (e && !strcmp(e, "cascade")) return false;
    if (e && !strcmp(e, "tau")) return m >= 2;
    return m >= 15;
}

void build_passes(PlanImpl &P) {
    const int m = P.m;
    const u64 n = P.n;
    const gf2e_tune &cfg = P.cfg;
    const u64 TILE = (u64)1 << cfg.fft_tile_log;
    auto choose = [&](u64 CH, u64 NS) { return choose_c(CH, NS, cfg); };
    auto mk = [&](u64 CH, u64 NS, u32 C) { return make_pass(CH, NS, C, n, cfg); };
    // deep depth L0: smallest L0 at which n >> L0 rows x C columns fit
    int L0 = 0;
    u32 Cd = 0;
    for (L0 = 0; L0 <= m; L0++) {
        u64 rows = n >> L0;
        if (rows > TILE) continue;
        Cd = choose((u64)1 << L0, rows);
        if (Cd) break;
    }
    if (L0 > m - 1) L0 = m - 1;            // n <= 2: degenerate
    if (m == 1) L0 = 0;
    if (!Cd) Cd = 1;
    std::vector<Pass> fwd, inv;
    const bool tau = use_tau_levels(m);
    if (tau) {
        // cascade levels (a = M - 2) grouped greedily into tile passes whose
        // rows span the index bits every level of the group touches; the
        // wider tau levels stream over HBM one at a time
        int cascade_bits = 0;
        for (int k = 2; k <= cfg.fft_tile_log; k++)
            if (choose((u64)1 << std::max(0, m - k), (u64)1 << k)) cascade_bits = k;
        cascade_bits = std::min(cascade_bits, 10);
        std::vector<std::pair<int, int>> lv;
        tau_levels(0, m, std::max(cascade_bits, 2), lv);
        auto fits = [&](int lo, int hi) {
            return hi - lo <= cfg.fft_tile_log &&
                   choose((u64)1 << lo, (u64)1 << (hi - lo)) != 0;
        };
        auto flush = [&](int lo, int hi, const std::vector<std::pair<int, int>> &g) {
            if (g.empty()) return;
            const u64 CH = (u64)1 << lo, NS = (u64)1 << (hi - lo);
            Pass pf = mk(CH, NS, choose(CH, NS));
            Pass pi = pf;
            for (const auto &o : g) pf.ops[pf.nops++] = mkop(TAY_F, (u32)(o.second - lo), 0);
            for (size_t k = g.size(); k-- > 0;)
                pi.ops[pi.nops++] = mkop(TAY_I, (u32)(g[k].second - lo), 0);
            fwd.push_back(pf);
            inv.push_back(pi);
        };
        std::vector<std::pair<int, int>> grp;
        int glo = 0, ghi = 0;
        for (const auto &o : lv) {
            const int M = o.first, a = o.second;
            if (M - a != 2 || !fits(a, M)) {
                flush(glo, ghi, grp);
                grp.clear();
                Pass ps;
                memset(&ps, 0, sizeof ps);
                ps.stream = 1;
                ps.sM = (u32)M;
                ps.sA = (u32)a;
                fwd.push_back(ps);
                inv.push_back(ps);
                continue;
            }
            if (!grp.empty()) {
                const int lo = std::min(glo, a), hi = std::max(ghi, M);
                if ((int)grp.size() < MAXOPS && fits(lo, hi)) {
                    glo = lo;
                    ghi = hi;
                    grp.push_back(o);
                    continue;
                }
                flush(glo, ghi, grp);
                grp.clear();
            }
            glo = a;
            ghi = M;
            grp.push_back(o);
        }
        flush(glo, ghi, grp);
    }
    // Taylor depths 0..L0-1, grouped levels
    for (int L = 0; !tau && L < L0 && L <= m - 2; L++) {
        int b_hi = m - L;
        while (b_hi >= 2) {
            int best_lo = b_hi;
            for (int b_lo = 2; b_lo <= b_hi; b_lo++) {
                u64 CH = (u64)1 << (b_lo - 2 + L);
                u64 NS = (u64)1 << (b_hi - b_lo + 2);
                if (b_hi - b_lo + 1 <= MAXOPS && choose(CH, NS)) { best_lo = b_lo; break; }
            }
            u64 CH = (u64)1 << (best_lo - 2 + L);
            u64 NS = (u64)1 << (b_hi - best_lo + 2);
            Pass pf = mk(CH, NS, choose(CH, NS));
            Pass pi = pf;
            for (int b = b_hi; b >= best_lo; b--) pf.ops[pf.nops++] = mkop(TAY_F, b - best_lo, 0);
            for (int b = best_lo; b <= b_hi; b++) pi.ops[pi.nops++] = mkop(TAY_I, b - best_lo, 0);
            fwd.push_back(pf);
            inv.push_back(pi);
            b_hi = best_lo - 1;
        }
    }
    // deep pass: Taylor depths L0..m-2 and butterflies m-1..L0
    {
        const int mp = m - L0;
        u64 CH = (u64)1 << L0, NS = n >> L0;
        Pass pf = mk(CH, NS, Cd);
        Pass pi = pf;
        for (int Lp = 0; !tau && Lp <= mp - 2; Lp++)
            for (int e = mp - 2; e >= Lp; e--) pf.ops[pf.nops++] = mkop(TAY_F, e, 0);
        for (int L = m - 1; L >= L0; L--) pf.ops[pf.nops++] = mkop(BF_F, L - L0, L);
        for (int L = L0; L <= m - 1; L++) pi.ops[pi.nops++] = mkop(BF_I, L - L0, L);
        for (int Lp = mp - 2; !tau && Lp >= 0; Lp--)
            for (int e = Lp; e <= mp - 2; e++) pi.ops[pi.nops++] = mkop(TAY_I, e, 0);
        fwd.push_back(pf);
        inv.push_back(pi);
    }
    // butterflies L0-1..0 in groups, built bottom-up
    std::vector<std::pair<int, int>> groups;   // (L_lo, L_hi)
    {
        int L_lo = 0;
        while (L_lo <= L0 - 1) {
            int best_hi = L_lo;
            for (int L_hi = L0 - 1; L_hi >= L_lo; L_hi--) {
                u64 CH = (u64)1 << L_lo, NS = (u64)1 << (L_hi - L_lo + 1);
                if (choose(CH, NS)) { best_hi = L_hi; break; }
            }
            groups.push_back({L_lo, best_hi});
            L_lo = best_hi + 1;
        }
    }
    for (size_t gi = groups.size(); gi-- > 0;) {          // forward: top group first
        int L_lo = groups[gi].first, L_hi = groups[gi].second;
        u64 CH = (u64)1 << L_lo, NS = (u64)1 << (L_hi - L_lo + 1);
        Pass pf = mk(CH, NS, choose(CH, NS));
        for (int L = L_hi; L >= L_lo; L--) pf.ops[pf.nops++] = mkop(BF_F, L - L_lo, L);
        fwd.push_back(pf);
    }
    std::vector<Pass> inv_b;
    for (size_t gi = 0; gi < groups.size(); gi++) {       // inverse: bottom group first
        int L_lo = groups[gi].first, L_hi = groups[gi].second;
        u64 CH = (u64)1 << L_lo, NS = (u64)1 << (L_hi - L_lo + 1);
        Pass pi = mk(CH, NS, choose(CH, NS));
        for (int L = L_lo; L <= L_hi; L++) pi.ops[pi.nops++] = mkop(BF_I, L - L_lo, L);
        inv_b.push_back(pi);
    }
    // inverse order: butterflies (bottom-up), deep pass, Taylor depths L0-1..0
    std::vector<Pass> inv_all = inv_b;
    inv_all.push_back(inv.back());
    for (size_t i = inv.size() - 1; i-- > 0;) inv_all.push_back(inv[i]);
    P.fwd = fwd;
    P.inv = inv_all;
    for (auto &p : P.fwd) merge_stages(p, cfg);
    for (auto &p : P.inv) merge_stages(p, cfg);
    for (auto &p : P.fwd) P.ntiles_fwd.push_back(pass_tiles(p, n));
    for (auto &p : P.inv) P.ntiles_inv.push_back(pass_tiles(p, n));
}

int run_passes(const PlanImpl &P, bool forward, u64 *f, const u32 *src32, u64 nchunks,
               cudaStream_t st, int batch = 1, Batch bt = Batch{0, 0, 0}) {
    const auto &ps = forward ? P.fwd : P.inv;
    const auto &nt = forward ? P.ntiles_fwd : P.ntiles_inv;
    if (src32 && !ps.empty() && ps[0].stream) {
        // the first pass streams: pack the operands first
        dim3 grid((unsigned)gf2e::grid_for(P.n, 256, 8), (unsigned)batch);
        k_pack_batch<<<grid, 256, 0, st>>>(src32, bt.sstride32, nchunks, bt.xor0, f, bt.fstride,
                                          P.n);
        GF2E_CHECK_LAUNCH("k_pack_batch");
        src32 = nullptr;
    }
    // 16-byte accesses in streaming levels need 16-byte aligned transforms
    const bool vec2 = ((uintptr_t)f % 16 == 0) && (batch == 1 || bt.fstride % 2 == 0);
    for (size_t i = 0; i < ps.size(); i++) {
        if (ps[i].stream) {
            const Pass &p = ps[i];
            const int V = (vec2 && p.sA >= 1) ? 2 : 1;
            dim3 grid((unsigned)gf2e::grid_for((P.n >> 1) / V, 256, 8), (unsigned)batch);
            if (V == 2)
                k_tau_stream<2><<<grid, 256, 0, st>>>(f, bt.fstride, P.n, (int)p.sM, (int)p.sA,
                                                      forward ? 1 : 0);
            else
                k_tau_stream<1><<<grid, 256, 0, st>>>(f, bt.fstride, P.n, (int)p.sM, (int)p.sA,
                                                      forward ? 1 : 0);
            GF2E_CHECK_LAUNCH("k_tau_stream");
            continue;
        }
        // many tiles per CTA: two tile buffers, one resident CTA per SM looping
        // over its tiles; otherwise one buffer and up to eight CTAs per SM
        const u64 sms = (u64)gf2e::sm_count();
        const bool db = nt[i] * (u64)batch >= 4 * sms;
        const size_t tile_bytes = ((size_t)1 << P.cfg.fft_tile_log) * sizeof(u64);
        const size_t smem = db ? 2 * tile_bytes : tile_bytes;
        const u64 per = std::max<u64>(1, (db ? sms : 8 * sms) / (u64)batch);
        dim3 grid((unsigned)std::min<u64>(nt[i], per), (unsigned)batch);
        const u32 *s32 = (i == 0) ? src32 : nullptr;
#define GF2E_FFT_LAUNCH(T, D) \
    k_fft_pass<T, D><<<grid, FFT_THREADS, smem, st>>>(f, P.tab, ps[i], nt[i], s32, nchunks, bt)
        switch (P.cfg.fft_tile_log * 2 + (db ? 1 : 0)) {
        case 22: GF2E_FFT_LAUNCH(11, false); break;
        case 23: GF2E_FFT_LAUNCH(11, true); break;
        case 24: GF2E_FFT_LAUNCH(12, false); break;
        case 25: GF2E_FFT_LAUNCH(12, true); break;
        case 26: GF2E_FFT_LAUNCH(13, false); break;
        default: GF2E_FFT_LAUNCH(13, true); break;
        }
#undef GF2E_FFT_LAUNCH
        GF2E_CHECK_LAUNCH("k_fft_pass");
    }
    return GF2E_OK;
}

}  // namespace

struct gf2e_fft_plan {
    PlanImpl impl;
};

namespace gf2e {

// the four 256-entry byte tables of W[t] (W is GF(2)-linear in t)
void twiddle_byte_tables(u64 *tab) {
    const u64 *b = basis_host();
    for (int k = 0; k < NTWTAB; k++)
        for (int v = 0; v < 256; v++) {
            u64 w = 0;
            for (int j = 0; j < 8; j++)
                if ((v >> j) & 1) w ^= b[8 * k + j + 1 < 64 ? 8 * k + j + 1 : 63];
            tab[k * 256 + v] = w;
        }
}

int twiddle_table_words() { return NTWTAB * 256; }

static int allow_tile_smem() {
    // set once per device; two threads racing here both set the same values
    static std::atomic<bool> done[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !done[dev].load(std::memory_order_acquire)) {
        cudaError_t e = cudaSuccess;
#define GF2E_FFT_ATTR(T, D, N)                                                              \
    if (e == cudaSuccess)                                                                   \
        e = cudaFuncSetAttribute(k_fft_pass<T, D>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                 (N) * (1 << T) * (int)sizeof(u64));
        GF2E_FFT_ATTR(11, false, 1) GF2E_FFT_ATTR(11, true, 2)
        GF2E_FFT_ATTR(12, false, 1) GF2E_FFT_ATTR(12, true, 2)
        GF2E_FFT_ATTR(13, false, 1) GF2E_FFT_ATTR(13, true, 2)
#undef GF2E_FFT_ATTR
        if (e != cudaSuccess) return cuda_status(e, "k_fft_pass smem attribute");
        done[dev].store(true, std::memory_order_release);
    }
    return GF2E_OK;
}

// knobs left at 0 take the size-dependent choice the autotuner makes on B200
// (tiles of 2^11 / 2^12 / 2^13 elements up to m = 17 / 21 / above, at least
// 2 / 4 / 8 contiguous columns up to m = 17 / 23 / above)
gf2e_tune resolve_by_size(gf2e_tune c, int m) {
    if (c.fft_tile_log == 0) c.fft_tile_log = m <= 17 ? 11 : (m <= 21 ? 12 : 13);
    if (c.fft_cmin == 0) c.fft_cmin = m <= 17 ? 2 : (m <= 23 ? 4 : 8);
    return c;
}

// plan whose passes read the caller's twiddle tables; no device allocation
int fft_plan_create_tables_cfg(int m, const u64 *tab_dev, const gf2e_tune &cfg,
                               gf2e_fft_plan **out) {
    if (m < 1 || m > 30) return invalid("FFT size exponent m=%d outside 1..30", m);
    if (!basis_host()) return invalid("Cantor basis construction failed");
    GF2E_TRY(allow_tile_smem());
    gf2e_fft_plan *p = new gf2e_fft_plan;
    p->impl.m = m;
    p->impl.n = (u64)1 << m;
    p->impl.tab = tab_dev;
    p->impl.cfg = resolve_by_size(cfg, m);
    build_passes(p->impl);
    *out = p;
    return GF2E_OK;
}

int fft_plan_create_tables(int m, const u64 *tab_dev, gf2e_fft_plan **out) {
    return fft_plan_create_tables_cfg(m, tab_dev, tune_current(), out);
}

// plan with its own twiddle tables and an explicit tuning
int fft_plan_create_cfg(int m, const gf2e_tune &cfg, gf2e_fft_plan **out) {
    if (m < 1 || m > 30) return invalid("FFT size exponent m=%d outside 1..30", m);
    if (!basis_host()) return invalid("Cantor basis construction failed");
    std::vector<u64> tab(NTWTAB * 256, 0);
    twiddle_byte_tables(tab.data());
    u64 *d_tab = nullptr;
    cudaError_t e = cudaMalloc(&d_tab, tab.size() * sizeof(u64));
    if (e == cudaSuccess)
        e = cudaMemcpy(d_tab, tab.data(), tab.size() * sizeof(u64), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(d_tab);
        return cuda_status(e, "fft plan twiddle tables");
    }
    int st = fft_plan_create_tables_cfg(m, d_tab, cfg, out);
    if (st != GF2E_OK) { cudaFree(d_tab); return st; }
    (*out)->impl.d_tab = d_tab;
    return GF2E_OK;
}

int fft_plan_create(int m, gf2e_fft_plan **out) {
    return fft_plan_create_cfg(m, tune_current(), out);
}

int fft_fwd_packed(const gf2e_fft_plan *plan, u64 *f, const u32 *src32, u64 nchunks,
                   cudaStream_t st) {
    return run_passes(plan->impl, true, f, src32, nchunks, st);
}

int fft_run(const gf2e_fft_plan *plan, bool forward, u64 *f, cudaStream_t st) {
    return run_passes(plan->impl, forward, f, nullptr, 0, st);
}

// `batch` transforms in one launch per pass: transform y at f + y*fstride,
// packed from src32 + y*sstride32 (chunk 0 XORed with xor0)
int fft_fwd_packed_batch(const gf2e_fft_plan *plan, u64 *f, u64 fstride, const u32 *src32,
                         u64 sstride32, u64 nchunks, u64 xor0, int batch, cudaStream_t st) {
    return run_passes(plan->impl, true, f, src32, nchunks, st, batch,
                      Batch{fstride, sstride32, xor0});
}

int fft_run_batch(const gf2e_fft_plan *plan, bool forward, u64 *f, u64 fstride, int batch,
                  cudaStream_t st) {
    return run_passes(plan->impl, forward, f, nullptr, 0, st, batch, Batch{fstride, 0, 0});
}

u64 fft_plan_n(const gf2e_fft_plan *plan) { return plan->impl.n; }

int pointwise(u64 *fa, const u64 *fb, u64 n, cudaStream_t st) {
    k_pointwise<<<grid_for(n, 256), 256, 0, st>>>(fa, fb, n);
    GF2E_CHECK_LAUNCH("k_pointwise");
    return GF2E_OK;
}

int overlap_add(const u64 *F, u64 nchunks, u64 *out, u64 ow, cudaStream_t st) {
    k_overlap_add<<<grid_for(ow, 256), 256, 0, st>>>(F, nchunks, out, ow);
    GF2E_CHECK_LAUNCH("k_overlap_add");
    return GF2E_OK;
}

int overlap_add_batch(const u64 *F, u64 fstride, u64 nchunks, u64 *out, u64 ostride, u64 ow,
                      int batch, cudaStream_t st) {
    int per = std::max(1, grid_for(ow, 256) / batch);
    k_overlap_add<<<dim3(per, batch), 256, 0, st>>>(F, nchunks, out, ow, fstride, ostride);
    GF2E_CHECK_LAUNCH("k_overlap_add batch");
    return GF2E_OK;
}

int mul_fft_m(u64 abits, u64 bbits) {
    u64 ca = (abits + 31) >> 5, cb = (bbits + 31) >> 5;
    int m = 1;
    while (((u64)1 << m) < ca + cb - 1) m++;
    return m;
}

// full product with a plan of size >= the needed one (gf2x_fft_mul_buf)
int mul(const gf2e_fft_plan *plan, const u64 *a, u64 abits, const u64 *b, u64 bbits,
        u64 *out, u64 *fa, u64 *fb, cudaStream_t st) {
    const u64 n = plan->impl.n;
    const u64 ca = (abits + 31) >> 5, cb = (bbits + 31) >> 5;
    if (abits == 0 || bbits == 0) return invalid("gf2e_mul: empty operand");
    if (ca + cb - 1 > n) return invalid("FFT too small: plan m=%d for %llu x %llu bits",
                                         plan->impl.m, (unsigned long long)abits,
                                         (unsigned long long)bbits);
    GF2E_TRY(fft_fwd_packed(plan, fa, reinterpret_cast<const u32 *>(a), ca, st));
    if (b == a && bbits == abits) {
        GF2E_TRY(pointwise(fa, fa, n, st));
    } else {
        GF2E_TRY(fft_fwd_packed(plan, fb, reinterpret_cast<const u32 *>(b), cb, st));
        GF2E_TRY(pointwise(fa, fb, n, st));
    }
    GF2E_TRY(fft_run(plan, false, fa, st));
    u64 ow = ((abits + bbits + 63) >> 6) + 1;
    return overlap_add(fa, ca + cb - 1, out, ow, st);
}

// plan cache shared by the batch API and the trinomial context
gf2e_fft_plan *cached_plan(int m) {
    static std::mutex mu;
    static std::map<std::pair<int, u64>, gf2e_fft_plan *> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    // plans are keyed by device, size and the tuning in force when made
    const gf2e_tune c = tune_current();
    const u64 key = (u64)m | ((u64)c.fft_tile_log << 8) | ((u64)c.fft_cmin << 16) |
                    ((u64)c.fft_taylor_lv << 32) | ((u64)c.fft_bfly_lv << 40);
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find({dev, key});
    if (it != cache.end()) return it->second;
    gf2e_fft_plan *p = nullptr;
    if (fft_plan_create(m, &p) != GF2E_OK) return nullptr;
    cache[{dev, key}] = p;
    return p;
}

}  // namespace gf2e

extern "C" {

int gf2e_cantor_basis(uint64_t *basis64, int *len) {
    const u64 *b = basis_host();
    if (!b) return gf2e::invalid("Cantor basis construction failed");
    if (basis64) memcpy(basis64, b, 64 * sizeof(u64));
    if (len) *len = 64;
    return GF2E_OK;
}

int gf2e_fft_plan_create(int m, gf2e_fft_plan **plan) {
    if (!plan) return gf2e::invalid("null plan pointer");
    return gf2e::fft_plan_create(m, plan);
}

int gf2e_fft_plan_destroy(gf2e_fft_plan *plan) {
    if (!plan) return GF2E_OK;
    cudaFree(plan->impl.d_tab);
    delete plan;
    return GF2E_OK;
}

int gf2e_fft_plan_m(const gf2e_fft_plan *plan) { return plan ? plan->impl.m : -1; }

int gf2e_fft_plan_passes(const gf2e_fft_plan *plan, int *fwd, int *inv) {
    if (!plan) return gf2e::invalid("null plan");
    if (fwd) *fwd = (int)plan->impl.fwd.size();
    if (inv) *inv = (int)plan->impl.inv.size();
    return GF2E_OK;
}

int gf2e_fft_fwd(const gf2e_fft_plan *plan, uint64_t *f_dev, void *stream) {
    if (!plan || !f_dev) return gf2e::invalid("gf2e_fft_fwd: null argument");
    return gf2e::fft_run(plan, true, f_dev, (cudaStream_t)stream);
}

int gf2e_fft_inv(const gf2e_fft_plan *plan, uint64_t *f_dev, void *stream) {
    if (!plan || !f_dev) return gf2e::invalid("gf2e_fft_inv: null argument");
    return gf2e::fft_run(plan, false, f_dev, (cudaStream_t)stream);
}

int gf2e_fft_pack(const uint64_t *a_dev, size_t nwords, uint64_t *f_dev, size_t nchunks,
                  size_t n, void *stream) {
    if (!a_dev || !f_dev || n == 0) return gf2e::invalid("gf2e_fft_pack: bad arguments");
    const u64 nc = std::min<u64>(nchunks, 2 * (u64)nwords);
    cudaStream_t st = (cudaStream_t)stream;
    k_pack_batch<<<gf2e::grid_for(n, 256), 256, 0, st>>>(
        reinterpret_cast<const u32 *>(a_dev), 0, nc, 0, f_dev, 0, n);
    GF2E_CHECK_LAUNCH("k_pack_batch");
    return GF2E_OK;
}

int gf2e_fft_pointwise(uint64_t *fa_dev, const uint64_t *fb_dev, size_t n, void *stream) {
    if (!fa_dev || !fb_dev) return gf2e::invalid("gf2e_fft_pointwise: null argument");
    if (n == 0) return GF2E_OK;
    return gf2e::pointwise(fa_dev, fb_dev, n, (cudaStream_t)stream);
}

int gf2e_fft_overlap_add(const uint64_t *f_dev, size_t nchunks, uint64_t *out_dev,
                         size_t owords, void *stream) {
    if (!f_dev || !out_dev) return gf2e::invalid("gf2e_fft_overlap_add: null argument");
    if (owords == 0) return GF2E_OK;
    return gf2e::overlap_add(f_dev, nchunks, out_dev, owords, (cudaStream_t)stream);
}

int gf2e_fft_twiddles(const gf2e_fft_plan *plan, uint64_t *W_host) {
    if (!plan || !W_host) return gf2e::invalid("gf2e_fft_twiddles: null argument");
    const u64 *b = basis_host();
    u64 half = plan->impl.n >> 1;
    if (half == 0) return GF2E_OK;
    W_host[0] = 0;
    for (u64 t = 1; t < half; t++) {
        int hb = 63 - __builtin_clzll(t);
        W_host[t] = W_host[t ^ (1ull << hb)] ^ b[hb + 1];
    }
    return GF2E_OK;
}

int gf2e_mul_fft_m(uint64_t abits, uint64_t bbits) { return gf2e::mul_fft_m(abits, bbits); }

size_t gf2e_mul_out_words(uint64_t abits, uint64_t bbits) {
    return (size_t)(((abits + bbits + 63) >> 6) + 1);
}

int gf2e_mul(const gf2e_fft_plan *plan, const uint64_t *a_dev, uint64_t abits,
             const uint64_t *b_dev, uint64_t bbits, uint64_t *out_dev, uint64_t *fa_dev,
             uint64_t *fb_dev, void *stream) {
    if (!plan || !a_dev || !b_dev || !out_dev || !fa_dev || !fb_dev)
        return gf2e::invalid("gf2e_mul: null argument");
    return gf2e::mul(plan, a_dev, abits, b_dev, bbits, out_dev, fa_dev, fb_dev,
                     (cudaStream_t)stream);
}

}  // extern "C"

namespace {
// words of batch workspace one job takes: two transforms of its size, or for
// a wrapped product two of the smaller size and its top-part scratch
size_t job_words(const gf2e_mul_job &j, gf2e::WrapMul *wm) {
    gf2e::WrapMul w;
    if (!getenv("GF2E_NO_WRAP") && gf2e::wrap_mul_plan(j.abits, j.bbits, w)) {
        if (wm) *wm = w;
        return 2 * (size_t)w.n + (size_t)w.per;
    }
    if (wm) wm->mb = 0;
    return 2 * ((size_t)1 << gf2e::mul_fft_m(j.abits, j.bbits));
}
}  // namespace

extern "C" {

int gf2e_mul_batch_workspace_size(const gf2e_mul_job *jobs, int njobs, size_t *bytes) {
    if (!jobs || njobs < 0 || !bytes) return gf2e::invalid("bad batch arguments");
    size_t tot = 0;
    for (int i = 0; i < njobs; i++) {
        if (jobs[i].abits == 0 || jobs[i].bbits == 0) return gf2e::invalid("empty operand in job %d", i);
        tot += job_words(jobs[i], nullptr) * sizeof(u64);
    }
    *bytes = tot;
    return GF2E_OK;
}

int gf2e_mul_batch(const gf2e_mul_job *jobs, int njobs, void *workspace, size_t ws_bytes,
                   void *stream) {
    size_t need = 0;
    GF2E_TRY(gf2e_mul_batch_workspace_size(jobs, njobs, &need));
    if (ws_bytes < need || (!workspace && need))
        return gf2e::invalid("gf2e_mul_batch: workspace %zu < %zu bytes", ws_bytes, need);
    cudaStream_t st = (cudaStream_t)stream;
    // fork onto a few internal streams so small products overlap large ones
    constexpr int NSTREAMS = 8;
    static thread_local cudaStream_t side[NSTREAMS] = {};
    static thread_local cudaEvent_t ev_side[NSTREAMS] = {};
    static thread_local cudaEvent_t ev_fork = nullptr;
    if (!ev_fork) {
        for (int i = 0; i < NSTREAMS; i++) {
            cudaStreamCreateWithFlags(&side[i], cudaStreamNonBlocking);
            cudaEventCreateWithFlags(&ev_side[i], cudaEventDisableTiming);
        }
        cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming);
    }
    cudaError_t e = cudaEventRecord(ev_fork, st);
    if (e != cudaSuccess) return gf2e::cuda_status(e, "batch fork");
    for (int i = 0; i < NSTREAMS; i++) cudaStreamWaitEvent(side[i], ev_fork, 0);
    // largest first, round-robin over streams
    std::vector<int> order(njobs);
    for (int i = 0; i < njobs; i++) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int x, int y) {
        return jobs[x].abits + jobs[x].bbits > jobs[y].abits + jobs[y].bbits;
    });
    std::vector<size_t> offs(njobs);
    std::vector<gf2e::WrapMul> wms(njobs);
    size_t off = 0;
    for (int i = 0; i < njobs; i++) {
        offs[i] = off;
        off += job_words(jobs[i], &wms[i]);
    }
    u64 *ws = (u64 *)workspace;
    for (int k = 0; k < njobs; k++) {
        int i = order[k];
        if (wms[i].mb) {                       // one size smaller, top part put back
            if (!gf2e::wrap_mul_plans(wms[i])) return gf2e::invalid("wrapped product plans");
            u64 *fa = ws + offs[i], *fb = fa + wms[i].n, *sc = fb + wms[i].n;
            GF2E_TRY(gf2e::mul_wrapped(wms[i], jobs[i].a_dev, jobs[i].abits, jobs[i].b_dev,
                                       jobs[i].bbits, jobs[i].out_dev, fa, fb, sc,
                                       side[k % NSTREAMS]));
            continue;
        }
        int m = gf2e::mul_fft_m(jobs[i].abits, jobs[i].bbits);
        gf2e_fft_plan *p = gf2e::cached_plan(m);
        if (!p) return gf2e::invalid("plan creation failed for m=%d", m);
        u64 *fa = ws + offs[i], *fb = fa + ((size_t)1 << m);
        GF2E_TRY(gf2e::mul(p, jobs[i].a_dev, jobs[i].abits, jobs[i].b_dev, jobs[i].bbits,
                           jobs[i].out_dev, fa, fb, side[k % NSTREAMS]));
    }
    for (int i = 0; i < NSTREAMS; i++) {
        cudaEventRecord(ev_side[i], side[i]);
        cudaStreamWaitEvent(st, ev_side[i], 0);
    }
    GF2E_CHECK_LAUNCH("gf2e_mul_batch");
    return GF2E_OK;
}

}  // extern "C"
