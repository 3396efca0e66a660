// gcd.cu -- batched GF(2)[x] gcd on the GPU, one CTA per pair.
//
// Replaces the CPU gcd that the reference runs on the interval accumulator
// (trinomial_scan.cu:64-141 GcdPool -> gf2_gcd.h:48-75 poly_gcd_naive /
// gf2_gcd_ntl.cpp:32-42 NTL).  Same contract as poly_gcd_naive: returns
// deg(gcd), 0 meaning gcd = 1 (and gcd(0, 0) = 0), and the gcd itself.
//
// Lehmer-style rounds.  From the top 64 bits of A and B (aligned at deg A)
// one thread runs Euclid reduction steps on the two windows, keeping the
// 2x2 transition matrix M of polynomials of degree <= 31, for as long as the
// window bits it decides on are exact (bits below the matrix degree are
// polluted by the unseen low parts).  Then the whole CTA applies M to the
// full operands, (A', B') = M (A, B), with carry-less 64x32 multiplies
// (masked integer products), about 32 degrees per round per operand.  A
// degree gap wider than the matrix allows is a single shift-XOR round.  The
// loop is bounded by deg A + deg B + 8 rounds (each round lowers the sum by
// at least one); exceeding it returns GF2E_ERR_TIMEOUT instead of looping.
#include "gf2e_internal.cuh"

#include <vector>

namespace {

constexpr int GCD_THREADS = 1024;

struct GcdDev {
    u64 *buf[4];          // A, B, and two scratch buffers, nw words each
    u64 nw;               // words per buffer
    u64 *g_out;           // destination for the gcd (g_cap words) or null
    u64 g_cap;
    long long deg;        // result
    int status;
};

// x (64 bits) times m (<= 32 bits): 96-bit result as (lo 64, hi 32)
GF2E_DEV void clmul64x32(const Masked &xl, const Masked &xh, const Masked &m, u64 &lo, u32 &hi) {
    u64 p0 = clmul_masked(xl, m), p1 = clmul_masked(xh, m);
    lo = p0 ^ (p1 << 32);
    hi = (u32)(p1 >> 32);
}

GF2E_DEV int deg64(u64 v) { return v ? 63 - __clzll(v) : -1; }

// 64-bit window of X at bit position pos (>= 0), zeros above the buffer
GF2E_DEV u64 win64(const u64 *X, u64 nw, u64 pos) {
    u64 i = pos >> 6;
    unsigned sh = (unsigned)(pos & 63);
    u64 a = i < nw ? X[i] : 0, b = i + 1 < nw ? X[i + 1] : 0;
    return funnel64(a, b, sh);
}

// plain Euclid on one-word operands
GF2E_DEV u64 gcd_word(u64 a, u64 b) {
    while (b) {
        int da = deg64(a), db = deg64(b);
        if (da < db) { u64 t = a; a = b; b = t; continue; }
        a ^= b << (da - db);
    }
    return a;
}

__global__ void __launch_bounds__(GCD_THREADS)
k_gcd_batch(GcdDev *__restrict__ jobs) {
    GcdDev &J = jobs[blockIdx.x];
    const int tid = threadIdx.x;
    const u64 nw = J.nw;
    __shared__ int s_ia, s_ib, s_ia2, s_ib2;     // buffer indices
    __shared__ long long s_da, s_db;
    __shared__ u64 s_top[4];                      // highest word ever written per buffer
    __shared__ int s_mode;                        // 0 matrix, 1 shift, 2 done
    __shared__ u32 s_m[4];                        // ma0, ma1, mb0, mb1
    __shared__ u64 s_k;                           // shift for mode 1
    __shared__ u32 s_hi[2][GCD_THREADS][4];       // neighbour carries
    __shared__ long long s_red[32];
    __shared__ int s_unit;                        // gcd found to be 1

    // initial degrees (block max of per-word degrees) and scratch zeroing
    for (int which = 0; which < 2; which++) {
        const u64 *X = J.buf[which];
        long long d = -1;
        for (u64 i = tid; i < nw; i += GCD_THREADS)
            if (X[i]) d = (long long)(i * 64 + 63 - __clzll(X[i]));
        for (int o = 16; o; o >>= 1) d = max(d, __shfl_down_sync(0xffffffffu, d, o));
        if ((tid & 31) == 0) s_red[tid >> 5] = d;
        __syncthreads();
        if (tid == 0) {
            long long m = -1;
            for (int w = 0; w < GCD_THREADS / 32; w++) m = max(m, s_red[w]);
            if (which == 0) s_da = m; else s_db = m;
        }
        __syncthreads();
    }
    for (u64 i = tid; i < nw; i += GCD_THREADS) { J.buf[2][i] = 0; J.buf[3][i] = 0; }
    if (tid == 0) {
        s_ia = 0; s_ib = 1; s_ia2 = 2; s_ib2 = 3;
        s_unit = 0;
        for (int i = 0; i < 4; i++) s_top[i] = nw - 1;
    }
    __syncthreads();

    const long long max_rounds = s_da + s_db + 8;
    long long round = 0;
    for (;; round++) {
        if (tid == 0) {
            long long da = s_da, db = s_db;
            if (da < db) {
                int t = s_ia; s_ia = s_ib; s_ib = t;
                t = s_ia2; s_ia2 = s_ib2; s_ib2 = t;
                long long x = da; da = db; db = x;
                s_da = da; s_db = db;
            }
            if (round > max_rounds) {
                s_mode = 2;
                J.status = GF2E_ERR_TIMEOUT;
            } else if (db < 0) {               // B = 0: gcd = A
                s_mode = 2;
                J.deg = da < 0 ? 0 : da;
                J.status = 0;
            } else if (db == 0) {              // B = 1
                s_mode = 2;
                J.deg = 0;
                J.status = 0;
                s_unit = 1;
            } else if (da < 64) {              // both fit one word
                u64 g = gcd_word(J.buf[s_ia][0], J.buf[s_ib][0]);
                J.buf[s_ia][0] = g;
                s_mode = 2;
                J.deg = deg64(g);
                J.status = 0;
            } else {
                const u64 *A = J.buf[s_ia], *B = J.buf[s_ib];
                const u64 lo = (u64)(da - 63);
                u64 a = win64(A, nw, lo), b = win64(B, nw, lo);
                u64 ma0 = 1, ma1 = 0, mb0 = 0, mb1 = 1;   // rows: A' = ma0 A + ma1 B
                int dga = 63, dgb = deg64(b), dma = 0, dmb = 0, steps = 0;
                for (int it = 0; it < 256; it++) {
                    if (dgb < 0) break;
                    if (dga < dgb) {
                        u64 t = a; a = b; b = t;
                        t = ma0; ma0 = mb0; mb0 = t;
                        t = ma1; ma1 = mb1; mb1 = t;
                        int x = dga; dga = dgb; dgb = x;
                        x = dma; dma = dmb; dmb = x;
                    }
                    // decide only on exact bits: positions >= the row's matrix degree
                    if (dgb < dmb || dga < dma) break;
                    const int k = dga - dgb;
                    const int ndm = max(dma, dmb + k);
                    if (ndm > 31) break;
                    a ^= b << k;
                    ma0 ^= mb0 << k;
                    ma1 ^= mb1 << k;
                    dma = ndm;
                    dga = deg64(a);
                    steps++;
                }
                if (steps == 0) {
                    s_mode = 1;
                    s_k = (u64)(da - db);
                } else {
                    s_mode = 0;
                    s_m[0] = (u32)ma0; s_m[1] = (u32)ma1; s_m[2] = (u32)mb0; s_m[3] = (u32)mb1;
                }
            }
        }
        __syncthreads();
        if (s_mode == 2) break;
        const int ia = s_ia, ib = s_ib, ia2 = s_ia2, ib2 = s_ib2;
        const u64 *A = J.buf[ia], *B = J.buf[ib];
        u64 *A2 = J.buf[ia2], *B2 = J.buf[ib2];
        const u64 wt = (u64)s_da >> 6;                       // top word of A and B
        const u64 wz = max(s_top[ia2], s_top[ib2]);          // stale words to clear
        if (s_mode == 1) {
            // A2 = A ^ (B << k); B unchanged (B2 gets a copy to keep roles uniform)
            const u64 k = s_k, ks = k >> 6;
            const unsigned kb = (unsigned)(k & 63);
            for (u64 w = tid; w <= wz; w += GCD_THREADS) {
                u64 va = 0, vb = 0;
                if (w <= wt) {
                    u64 hi = (w >= ks) ? B[w - ks] : 0;
                    u64 lo2 = (w >= ks + 1) ? B[w - ks - 1] : 0;
                    u64 sh = kb ? ((hi << kb) | (lo2 >> (64 - kb))) : hi;
                    va = A[w] ^ sh;
                    vb = B[w];
                }
                A2[w] = va;
                B2[w] = vb;
            }
        } else {
            const Masked m0 = mask32(s_m[0]), m1 = mask32(s_m[1]), m2 = mask32(s_m[2]),
                         m3 = mask32(s_m[3]);
            const u64 nblk = (wz + GCD_THREADS) / GCD_THREADS;
            for (u64 blk = 0; blk < nblk; blk++) {
                const u64 w = blk * GCD_THREADS + tid;
                u64 xa = (w <= wt) ? A[w] : 0, xb = (w <= wt) ? B[w] : 0;
                Masked al = mask32((u32)xa), ah = mask32((u32)(xa >> 32));
                Masked bl = mask32((u32)xb), bh = mask32((u32)(xb >> 32));
                u64 l0, l1, l2, l3;
                u32 h0, h1, h2, h3;
                clmul64x32(al, ah, m0, l0, h0);
                clmul64x32(bl, bh, m1, l1, h1);
                clmul64x32(al, ah, m2, l2, h2);
                clmul64x32(bl, bh, m3, l3, h3);
                const int par = blk & 1;
                s_hi[par][tid][0] = h0; s_hi[par][tid][1] = h1;
                s_hi[par][tid][2] = h2; s_hi[par][tid][3] = h3;
                __syncthreads();
                u32 c0 = 0, c1 = 0, c2 = 0, c3 = 0;            // carries from word w-1
                if (tid > 0) {
                    c0 = s_hi[par][tid - 1][0]; c1 = s_hi[par][tid - 1][1];
                    c2 = s_hi[par][tid - 1][2]; c3 = s_hi[par][tid - 1][3];
                } else if (blk > 0) {
                    c0 = s_hi[par ^ 1][GCD_THREADS - 1][0]; c1 = s_hi[par ^ 1][GCD_THREADS - 1][1];
                    c2 = s_hi[par ^ 1][GCD_THREADS - 1][2]; c3 = s_hi[par ^ 1][GCD_THREADS - 1][3];
                }
                if (w <= wz) {
                    A2[w] = l0 ^ l1 ^ (u64)c0 ^ (u64)c1;
                    B2[w] = l2 ^ l3 ^ (u64)c2 ^ (u64)c3;
                }
            }
        }
        __syncthreads();
        // new roles and degrees: scan down from the old top word (warp 0)
        if (tid < 32) {
            for (int which = 0; which < 2; which++) {
                const u64 *X = J.buf[which == 0 ? ia2 : ib2];
                long long d = -1;
                for (long long base = (long long)wt; base >= 0 && d < 0; base -= 32) {
                    long long i = base - tid;
                    u64 v = (i >= 0) ? X[i] : 0;
                    unsigned ball = __ballot_sync(0xffffffffu, v != 0);
                    if (ball) {
                        int lane = __ffs(ball) - 1;      // highest word = lowest lane
                        u64 vv = __shfl_sync(0xffffffffu, v, lane);
                        d = (base - lane) * 64 + 63 - __clzll(vv);
                    }
                }
                if (tid == 0) {
                    if (which == 0) s_da = d; else s_db = d;
                }
            }
            if (tid == 0) {
                // words above the new degrees are zero in the buffers just written
                s_top[ia2] = s_da > 0 ? ((u64)s_da >> 6) : 0;
                s_top[ib2] = s_db > 0 ? ((u64)s_db >> 6) : 0;
                int t = s_ia; s_ia = s_ia2; s_ia2 = t;
                t = s_ib; s_ib = s_ib2; s_ib2 = t;
            }
        }
        __syncthreads();
    }
    // deliver the gcd (in buffer s_ia) when it fits the caller's capacity
    __syncthreads();
    if (J.status == 0 && J.g_out) {
        const u64 gw = (u64)J.deg / 64 + 1;
        const u64 *G = J.buf[s_ia];
        if (gw <= J.g_cap)
            for (u64 i = tid; i < J.g_cap; i += GCD_THREADS)
                J.g_out[i] = s_unit ? (i == 0 ? 1ull : 0ull) : ((i < gw) ? G[i] : 0);
    }
}

}  // namespace

extern "C" {

int gf2e_gcd_workspace_size(const gf2e_gcd_job *jobs, int njobs, size_t *bytes) {
    if (!jobs || njobs < 1 || !bytes) return gf2e::invalid("gf2e_gcd: bad job list");
    size_t tot = ((size_t)njobs * sizeof(GcdDev) + 255) & ~(size_t)255;
    for (int i = 0; i < njobs; i++) {
        u64 bits = jobs[i].abits > jobs[i].bbits ? jobs[i].abits : jobs[i].bbits;
        size_t nw = (size_t)((bits + 63) >> 6) + 1;
        tot += 4 * nw * 8;
    }
    *bytes = tot;
    return GF2E_OK;
}

int gf2e_gcd_batch(const gf2e_gcd_job *jobs, int njobs, int64_t *deg_host, void *workspace,
                   size_t ws_bytes, void *stream) {
    size_t need = 0;
    GF2E_TRY(gf2e_gcd_workspace_size(jobs, njobs, &need));
    if (!workspace || ws_bytes < need || !deg_host)
        return gf2e::invalid("gf2e_gcd_batch: workspace %zu < %zu bytes", ws_bytes, need);
    if (njobs > 65535) return gf2e::invalid("gf2e_gcd_batch: at most 65535 jobs");
    cudaStream_t st = (cudaStream_t)stream;
    std::vector<GcdDev> host(njobs);
    char *ws = (char *)workspace;
    GcdDev *djobs = (GcdDev *)ws;
    size_t off = ((size_t)njobs * sizeof(GcdDev) + 255) & ~(size_t)255;
    for (int i = 0; i < njobs; i++) {
        const gf2e_gcd_job &j = jobs[i];
        if (!j.a_dev || !j.b_dev) return gf2e::invalid("gf2e_gcd_batch: null operand in job %d", i);
        u64 bits = j.abits > j.bbits ? j.abits : j.bbits;
        u64 nw = ((bits + 63) >> 6) + 1;
        GcdDev &g = host[i];
        for (int b = 0; b < 4; b++) { g.buf[b] = (u64 *)(ws + off); off += nw * 8; }
        g.nw = nw;
        g.g_out = j.g_dev;
        g.g_cap = j.g_cap_words;
        g.deg = -1;
        g.status = GF2E_ERR_INTERNAL;
        // operands into the working buffers, zero-extended
        size_t wa = (size_t)((j.abits + 63) >> 6), wb = (size_t)((j.bbits + 63) >> 6);
        cudaError_t e = cudaMemsetAsync(g.buf[0], 0, nw * 8, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(g.buf[1], 0, nw * 8, st);
        if (e == cudaSuccess && wa) e = cudaMemcpyAsync(g.buf[0], j.a_dev, wa * 8, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess && wb) e = cudaMemcpyAsync(g.buf[1], j.b_dev, wb * 8, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return gf2e::cuda_status(e, "gcd operand staging");
    }
    cudaError_t e = cudaMemcpyAsync(djobs, host.data(), njobs * sizeof(GcdDev),
                                    cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return gf2e::cuda_status(e, "gcd job upload");
    k_gcd_batch<<<njobs, GCD_THREADS, 0, st>>>(djobs);
    GF2E_CHECK_LAUNCH("k_gcd_batch");
    e = cudaMemcpyAsync(host.data(), djobs, njobs * sizeof(GcdDev), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return gf2e::cuda_status(e, "gcd results");
    int worst = GF2E_OK;
    for (int i = 0; i < njobs; i++) {
        deg_host[i] = host[i].deg;
        if (host[i].status != GF2E_OK) {
            worst = host[i].status;
            gf2e::set_error("gcd job %d: status %d", i, host[i].status);
        }
    }
    return worst;
}

}  // extern "C"
