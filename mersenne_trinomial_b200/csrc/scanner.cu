// scanner.cu -- the resident, steppable deep-scan engine behind gf2e_scan
// and the serving loop.
//
// One scanner serves one r.  It owns device state for `slots` s values
// (F, scratch, ACC, the two transform buffers, the product, the trinomial),
// a queue of submitted s values (each with its own k0, maxd and interval
// policy, tagged by the caller), and a list of finished results.  A step
// advances every resident s by one degree with batched launches (squaring,
// two packed transforms, pointwise product, inverse, overlap-add, fold),
// runs one batched gcd for the s whose interval ends, resolves hits on the
// host, retires finished s and refills their slots from the queue (or
// compacts the slots when the queue is empty).  Per-s state stays on the
// device between steps, so different jobs' s values share every launch.
//
// Blocked mode (block size m > 1) is the multi-level blocking DDF of the
// reference's tsfactor (tsfactor.cu:1-27, 71-126, 296-365; after gf2x
// factor.cpp): per s it keeps h[j] = e_{j+1}(y_0..y_{m-1}), the elementary
// symmetric functions of the Frobenius iterates y_t = x^(2^(i+t)) mod T of
// the current block of degrees [i, i+m-1].  Then
//   C = x^m + h[0] x^(m-1) + ... + h[m-1] = prod_t (x + x^(2^(i+t)))  (mod T)
// is one shift-XOR pass (Horner at x), ACC *= C is one modmul per block, and
// h[j] <- h[j]^(2^m) advances the block (Frobenius commutes with e_k): per
// degree m squarings and 1/m modmul instead of one modmul.  ACC after q
// blocks is the same residue as after q*m single degrees, so the gcds and
// results are the per-degree scanner's.  Initial h for the block at degree 0
// follows E_j(X) = (X + x) E_{j-1}^(2)(X) with E_j = prod_{t<j} (X + x^(2^t))
// (squarings and multiplications by x only); it is then advanced by k0 + 1
// Frobenius steps.
#include "gf2e_internal.cuh"
#include "polyhost.h"
#include "wrapmul.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <deque>
#include <vector>

namespace gf2e {
int trin_square_states(const u64 *in, u64 *out, size_t stride, int nstates, u64 r,
                       const u64 *s_dev, cudaStream_t st);
int frobenius_states(u64 *a, u64 *b, size_t stride, int nstates, u64 r, const u64 *s_dev,
                     u64 k, cudaStream_t st, u64 s_uniform);
int trin_set_const(u64 *states, size_t stride, int nstates, u64 r, u64 w0, cudaStream_t st);
int trin_reduce_batch(const u64 *P, size_t pstride, size_t pw, u64 L, u64 *out, size_t ostride,
                      u64 r, const u64 *s_dev, int batch, cudaStream_t st);
int fft_fwd_packed_batch(const gf2e_fft_plan *plan, u64 *f, u64 fstride, const u32 *src32,
                         u64 sstride32, u64 nchunks, u64 xor0, int batch, cudaStream_t st);
int fft_run_batch(const gf2e_fft_plan *plan, bool forward, u64 *f, u64 fstride, int batch,
                  cudaStream_t st);
int overlap_add_batch(const u64 *F, u64 fstride, u64 nchunks, u64 *out, u64 ostride, u64 ow,
                      int batch, cudaStream_t st);
int pointwise(u64 *fa, const u64 *fb, u64 n, cudaStream_t st);
int mul_fft_m(u64 abits, u64 bbits);
gf2e_fft_plan *cached_plan(int m);
u64 fft_plan_n(const gf2e_fft_plan *plan);
}  // namespace gf2e

struct gf2e_scanner {
    struct Job { u64 s, k0, maxd, L0, Lmax, tag; gf2e_sched sched; };
    struct Slot { Job job; u64 k, iv, L; };
    struct Done { gf2e_scan_result res; u64 tag; std::vector<u64> mask; };

    u64 r = 0;
    int B = 0;
    size_t nw = 0, stride = 0, tw = 0, ow = 0, pstride = 0, gcap = 0;
    u64 n = 0, nchunks = 0;
    gf2e_fft_plan *plan = nullptr;
    u64 *dmem = nullptr, *F = nullptr, *Fs = nullptr, *ACC = nullptr, *FA = nullptr,
        *FB = nullptr, *P = nullptr, *T = nullptr, *sdev = nullptr, *G = nullptr;
    void *gws = nullptr;
    size_t gws_bytes = 0, dmem_bytes = 0;
    std::deque<Job> queue;
    std::vector<Slot> slot;
    int nact = 0;
    std::deque<Done> done;
    std::vector<u64> shost, thost, ghost;
    std::vector<int64_t> degs;
    std::vector<gf2e_gcd_job> jobs;
    u64 degree_steps = 0, sd_pairs = 0;
    u64 gcds = 0;                 // interval gcds run, and their host wall time
    double gcd_seconds = 0;
    // the per-degree launches (squaring, transforms, products, folds) are
    // replayed from CUDA graphs, one per (resident count, F buffer)
    cudaStream_t own = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    struct GraphKey { int nact; const u64 *F; };
    std::vector<std::pair<GraphKey, cudaGraphExec_t>> graphs;
    bool use_graphs = true;
    int gcd_parallel = 64;        // half-gcds per lockstep batch at interval ends (large r)
    // blocked mode: m residues h per slot (slot j's at H + (j*m + t)*stride),
    // their squaring scratch, the block product C per slot, s per h state
    int m = 1;
    u64 *H = nullptr, *HS = nullptr, *C = nullptr, *sH = nullptr;
    std::vector<u64> shH;
    gf2e_sched sched{GF2E_SCHED_DOUBLING, 0, 0, 0.0, 0};   // for jobs submitted next
    // r-bit products one transform size smaller, the wrapped part put back
    bool wrap = false;
    gf2e::WrapMul wm;
    u64 *WS = nullptr;
};

// operands of at least this many bits take the half-gcd (hgcd.cu) at
// interval ends; smaller ones the quadratic batched gcd (gcd.cu)
constexpr u64 GCD_LARGE_BITS = 1ull << 19;
// device words one member of a lockstep half-gcd batch draws from the gcd
// pool, per operand word (its high-water mark: 1.52 GB at r = 136279841)
constexpr size_t HGCD_WORDS_PER_WORD = 90;

namespace gf2e {

// Interval schedules (the gcd cadence of the deep scan), in degrees.
//   DOUBLING: L0, 2 L0, 4 L0, ... capped at Lmax (trinomial_scan.cu:379-381)
//   LINEAR:   q0, 2 q0, 3 q0, ... blocks of m degrees (tsfactor.cu:858)
//   OPT:      tsfactor's Euler-optimal widths (tsfactor.cu:837-891): with the
//             survival law S(k) = (16/9)/k and gcd cost G degrees of scanning,
//             stationarity of sum S(k_{j-1}) (w_j + G) gives
//             w' = w k / (k - w) - G, kept non-decreasing and at least
//             (rho - 1) k; the first width minimises that cost over 96
//             candidate first ends.
// qcap > 0 caps an interval at qcap blocks (tsfactor --Zq) in LINEAR and OPT.
u64 sched_first(const gf2e_sched &q, u64 m, u64 k_start, u64 L0) {
    if (q.mode == GF2E_SCHED_DOUBLING) return L0;
    u64 blocks = 0;
    if (q.mode == GF2E_SCHED_LINEAR) {
        blocks = q.q0;
    } else {
        const double G = (double)q.G, C = 16.0 / 9.0, grow = q.rho - 1.0;
        const u64 k0 = k_start;
        u64 lo = (u64)(1.02 * std::sqrt((double)k0 * G)) + 1;
        if (lo <= k0) lo = k0 + m;
        double best = 1e300;
        u64 best_k1 = 0;
        for (int i = 0; i < 96; i++) {
            const u64 k1 = lo + (u64)((double)lo * 0.06 * i);
            double cost = 0, kp = (double)k0, kc = (double)k1;
            for (int j = 0; j < 200 && kp < 4e18; j++) {
                cost += (C / kp) * ((kc - kp) + G);
                double w = kc * kc / kp - G - kc;
                w = std::max(w, kc - kp);
                w = std::max(w, grow * kc);
                kp = kc;
                kc += w;
                if (kp > 1e14) break;
            }
            if (cost < best) {
                best = cost;
                best_k1 = k1;
            }
        }
        const u64 w = best_k1 > k0 ? best_k1 - k0 : m;
        blocks = (w + m - 1) / m;
    }
    blocks = std::max<u64>(blocks, 1);
    if (q.qcap) blocks = std::min(blocks, q.qcap);
    return blocks * m;
}

// width after an interval of `cur` degrees that ended at degree k_end
u64 sched_next(const gf2e_sched &q, u64 m, u64 cur, u64 k_end, u64 Lmax) {
    if (q.mode == GF2E_SCHED_DOUBLING) return std::min(2 * cur, Lmax);
    u64 blocks;
    if (q.mode == GF2E_SCHED_LINEAR) {
        blocks = cur / m + q.q0;
    } else {
        const double k = (double)k_end, w = (double)cur;
        double wn = k > w ? w * k / (k - w) - (double)q.G : w;
        wn = std::max(wn, w);
        wn = std::max(wn, (q.rho - 1.0) * k);
        wn = std::min(wn, 4e18);
        blocks = ((u64)wn + m - 1) / m;
    }
    blocks = std::max<u64>(blocks, 1);
    if (q.qcap) blocks = std::min(blocks, q.qcap);
    return blocks * m;
}

int sched_check(const gf2e_sched *q) {
    if (!q) return invalid("null schedule");
    if (q->mode == GF2E_SCHED_DOUBLING) return GF2E_OK;
    if (q->mode == GF2E_SCHED_LINEAR) return q->q0 >= 1 ? GF2E_OK : invalid("linear schedule: q0 >= 1");
    if (q->mode == GF2E_SCHED_OPT)
        return (q->G >= 1 && q->rho > 1.0) ? GF2E_OK : invalid("opt schedule: G >= 1 and rho > 1");
    return invalid("schedule mode %d", q->mode);
}

}  // namespace gf2e

namespace {

struct Geometry {
    size_t nw, stride, tw, ow, pstride, gcap;
    u64 n, nchunks;
    int m;
    bool wrap;
    gf2e::WrapMul wm;
};

Geometry geometry(u64 r) {
    Geometry g;
    g.nw = (size_t)((r + 63) >> 6);
    g.stride = g.nw + (g.nw & 1);
    g.tw = (size_t)((r + 1 + 63) >> 6);
    g.m = gf2e::mul_fft_m(r, r);
    g.wrap = !getenv("GF2E_NO_WRAP") && gf2e::wrap_mul_plan(r, r, g.wm);
    if (g.wrap) g.m = g.wm.mb;
    g.n = (u64)1 << g.m;
    g.nchunks = (r + 31) >> 5;
    g.ow = (size_t)(((2 * r + 63) >> 6) + 1);
    g.pstride = g.ow + (g.ow & 1);
    g.gcap = std::min<size_t>(g.tw, 4096);
    return g;
}

size_t device_words(const Geometry &g, int B, int m = 1) {
    size_t w = 3 * g.stride * B + 2 * g.n * B + g.pstride * B + g.tw * B + B + g.gcap * B;
    if (m > 1) w += 2 * (size_t)m * g.stride * B + g.stride * B + (size_t)m * B;
    if (g.wrap) w += (size_t)g.wm.per * B;
    return w;
}

// word w of x * v mod x^r + x^s + 1 (v a residue, bits >= r zero)
__device__ __forceinline__ u64 mulx_word(const u64 *v, u64 r, u64 s, u64 w) {
    const u64 a = v[w], b = w ? v[w - 1] : 0;
    u64 out = (a << 1) | (b >> 63);
    const u64 wrap = (v[(r - 1) >> 6] >> ((r - 1) & 63)) & 1;      // coefficient of x^(r-1)
    if (w == (r >> 6)) out &= ~(1ull << (r & 63));                  // x^r -> x^s + 1
    if (w == 0) out ^= wrap;
    if (w == (s >> 6)) out ^= wrap << (s & 63);
    return out;
}

// one step of E_j = (X + x) E_{j-1}^(2): h[t] <- S[t] + x S[t-1] (+ x at
// t = 0) for t < j, where S[t] = h[t]^2 (S[j-1] = 0); state t = blockIdx.y
__global__ void k_esym_step(u64 *__restrict__ Hs, const u64 *__restrict__ Sq, size_t stride,
                            int j, u64 nw, u64 r, u64 s) {
    const int t = blockIdx.y;
    u64 *out = Hs + (size_t)t * stride;
    const u64 *cur = Sq + (size_t)t * stride, *prev = Sq + (size_t)(t - 1) * stride;
    for (u64 w = (u64)blockIdx.x * blockDim.x + threadIdx.x; w < nw;
         w += (u64)gridDim.x * blockDim.x) {
        u64 v = (t < j - 1) ? cur[w] : 0;
        if (t >= 1) v ^= mulx_word(prev, r, s, w);
        if (t == 0 && w == 0) v ^= 2;
        out[w] = v;
    }
}

// C = x^m + sum_t h[t] x^(m-1-t), bits >= r dropped here (folded by
// k_horner_fold); slot = blockIdx.y
__global__ void k_horner(const u64 *__restrict__ H, size_t stride, int m, u64 *__restrict__ C,
                         u64 nw, u64 r) {
    const int y = blockIdx.y;
    const u64 *h0 = H + (size_t)y * m * stride;
    u64 *c = C + (size_t)y * stride;
    const u64 topmask = (r & 63) ? ((1ull << (r & 63)) - 1) : ~0ull;
    for (u64 w = (u64)blockIdx.x * blockDim.x + threadIdx.x; w < nw;
         w += (u64)gridDim.x * blockDim.x) {
        u64 acc = 0;
        for (int t = 0; t < m; t++) {
            const u64 *h = h0 + (size_t)t * stride;
            const unsigned sh = (unsigned)(m - 1 - t);
            const u64 a = h[w], b = w ? h[w - 1] : 0;
            acc ^= sh ? ((a << sh) | (b >> (64 - sh))) : a;
        }
        if (w == nw - 1) acc &= topmask;
        if (w == ((u64)m >> 6)) acc ^= 1ull << (m & 63);
        c[w] = acc;
    }
}

// the bits of sum_t h[t] x^(m-1-t) at x^(r+e), e <= m-2, folded as
// x^(r+e) = x^(s+e) + x^e (one thread per slot)
__global__ void k_horner_fold(const u64 *__restrict__ H, size_t stride, int m, u64 *C, u64 r,
                              const u64 *__restrict__ s_dev) {
    const int y = blockIdx.x;
    if (threadIdx.x != 0) return;
    const u64 *h0 = H + (size_t)y * m * stride;
    u64 *c = C + (size_t)y * stride;
    const u64 s = s_dev[y];
    u64 O = 0;                                   // bit e = coefficient of x^(r+e)
    for (int t = 0; t < m - 1; t++) {
        const unsigned sh = (unsigned)(m - 1 - t);     // h[t] bits [r-sh, r) move to [r, r+sh)
        const u64 p = r - sh, i = p >> 6;
        const unsigned b = (unsigned)(p & 63);
        u64 win = h0[(size_t)t * stride + i] >> b;
        if (b && ((r - 1) >> 6) > i) win |= h0[(size_t)t * stride + i + 1] << (64 - b);
        O ^= win & ((1ull << sh) - 1);
    }
    if (!O) return;
    c[0] ^= O;
    const u64 sw = s >> 6;
    const unsigned sb = (unsigned)(s & 63);
    c[sw] ^= O << sb;
    if (sb) c[sw + 1] ^= O >> (64 - sb);
}

int load_slot(gf2e_scanner &S, int j, const gf2e_scanner::Job &job, cudaStream_t st) {
    std::fill(S.thost.begin(), S.thost.end(), 0);
    S.thost[0] |= 1;
    S.thost[job.s >> 6] |= 1ull << (job.s & 63);
    S.thost[S.r >> 6] |= 1ull << (S.r & 63);
    S.shost[j] = job.s;
    cudaError_t e = cudaMemcpyAsync(S.T + S.tw * j, S.thost.data(), S.tw * 8,
                                    cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(S.sdev + j, &S.shost[j], 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);      // host staging reused
    if (e != cudaSuccess) return gf2e::cuda_status(e, "scanner slot load");
    GF2E_TRY(gf2e::trin_set_const(S.ACC + S.stride * j, S.stride, 1, S.r, 1, st));
    if (S.m > 1) {
        // h for the block at degree 0, then k0 + 1 Frobenius steps
        const int m = S.m;
        u64 *Hj = S.H + (size_t)j * m * S.stride, *HSj = S.HS + (size_t)j * m * S.stride;
        const u64 *sHj = S.sH + (size_t)j * m;
        for (int t = 0; t < m; t++) S.shH[(size_t)j * m + t] = job.s;
        e = cudaMemcpyAsync(S.sH + (size_t)j * m, S.shH.data() + (size_t)j * m, (size_t)m * 8,
                            cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return gf2e::cuda_status(e, "scanner block slot load");
        const int gx = std::max(1, gf2e::grid_for(S.nw, 256) / m);
        for (int jj = 1; jj <= m; jj++) {
            if (jj > 1)
                GF2E_TRY(gf2e::trin_square_states(Hj, HSj, S.stride, jj - 1, S.r, sHj, st));
            k_esym_step<<<dim3(gx, jj), 256, 0, st>>>(Hj, HSj, S.stride, jj, S.nw, S.r, job.s);
            GF2E_CHECK_LAUNCH("k_esym_step");
        }
        GF2E_TRY(gf2e::frobenius_states(Hj, HSj, S.stride, m, S.r, sHj, job.k0 + 1, st, 0));
        S.slot[j] = gf2e_scanner::Slot{
            job, job.k0, job.k0, gf2e::sched_first(job.sched, (u64)m, job.k0 + 1, job.L0)};
        return GF2E_OK;
    }
    GF2E_TRY(gf2e::trin_set_const(S.F + S.stride * j, S.stride, 1, S.r, 2, st));
    GF2E_TRY(gf2e::frobenius_states(S.F + S.stride * j, S.Fs + S.stride * j, S.stride, 1, S.r,
                                    S.sdev + j, job.k0, st, 0));
    S.slot[j] = gf2e_scanner::Slot{job, job.k0, job.k0,
                                   gf2e::sched_first(job.sched, 1, job.k0 + 1, job.L0)};
    return GF2E_OK;
}

int move_slot(gf2e_scanner &S, int to, int from, cudaStream_t st) {
    cudaError_t e = cudaMemcpyAsync(S.F + S.stride * to, S.F + S.stride * from, S.stride * 8,
                                    cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(S.ACC + S.stride * to, S.ACC + S.stride * from, S.stride * 8,
                            cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(S.T + S.tw * to, S.T + S.tw * from, S.tw * 8,
                            cudaMemcpyDeviceToDevice, st);
    S.shost[to] = S.shost[from];
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(S.sdev + to, &S.shost[to], 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && S.m > 1) {
        const size_t mw = (size_t)S.m * S.stride;
        e = cudaMemcpyAsync(S.H + to * mw, S.H + from * mw, mw * 8, cudaMemcpyDeviceToDevice, st);
        for (int t = 0; t < S.m; t++) S.shH[(size_t)to * S.m + t] = S.shost[to];
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(S.sH + (size_t)to * S.m, S.shH.data() + (size_t)to * S.m,
                                (size_t)S.m * 8, cudaMemcpyHostToDevice, st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    S.slot[to] = S.slot[from];
    return gf2e::cuda_status(e, "scanner compaction");
}

int fill_slots(gf2e_scanner &S, cudaStream_t st) {
    while (S.nact < S.B && !S.queue.empty()) {
        gf2e_scanner::Job job = S.queue.front();
        S.queue.pop_front();
        GF2E_TRY(load_slot(S, S.nact, job, st));
        S.nact++;
    }
    return GF2E_OK;
}

// the product's last step: P = ACC * B from the inverse transform in FA
// (overlap-add, and for wrapped products the top part put back)
int product_tail(gf2e_scanner &S, int na, const u64 *B, cudaStream_t st) {
    if (S.wrap)
        return gf2e::wrap_mul_finish(S.wm, S.FA, S.n, S.ACC, S.stride, B, S.stride, S.P,
                                     S.pstride, S.ow, na, S.WS, st);
    return gf2e::overlap_add_batch(S.FA, S.n, 2 * S.nchunks - 1, S.P, S.pstride, S.ow, na, st);
}

// the launches of one degree for `na` resident s (F -> Fs squared; the
// product then reads Fs, which becomes F)
int degree_kernels(gf2e_scanner &S, int na, u64 *F, u64 *Fs, cudaStream_t st) {
    GF2E_TRY(gf2e::trin_square_states(F, Fs, S.stride, na, S.r, S.sdev, st));
    GF2E_TRY(gf2e::fft_fwd_packed_batch(S.plan, S.FA, S.n, reinterpret_cast<const u32 *>(S.ACC),
                                        2 * S.stride, S.nchunks, 0, na, st));
    GF2E_TRY(gf2e::fft_fwd_packed_batch(S.plan, S.FB, S.n, reinterpret_cast<const u32 *>(Fs),
                                        2 * S.stride, S.nchunks, 2, na, st));
    GF2E_TRY(gf2e::pointwise(S.FA, S.FB, S.n * na, st));
    GF2E_TRY(gf2e::fft_run_batch(S.plan, false, S.FA, S.n, na, st));
    GF2E_TRY(product_tail(S, na, Fs, st));
    GF2E_TRY(gf2e::trin_reduce_batch(S.P, S.pstride, S.ow, 2 * S.r - 1, S.ACC, S.stride, S.r,
                                     S.sdev, na, st));
    return GF2E_OK;
}

// the launches of one block of m degrees for `na` resident s: C by Horner,
// ACC *= C mod T, then every h squared m times (m even: back in H)
int block_kernels(gf2e_scanner &S, int na, cudaStream_t st) {
    const int m = S.m;
    const int gx = std::max(1, gf2e::grid_for(S.nw, 256) / na);
    k_horner<<<dim3(gx, na), 256, 0, st>>>(S.H, S.stride, m, S.C, S.nw, S.r);
    GF2E_CHECK_LAUNCH("k_horner");
    k_horner_fold<<<na, 32, 0, st>>>(S.H, S.stride, m, S.C, S.r, S.sdev);
    GF2E_CHECK_LAUNCH("k_horner_fold");
    GF2E_TRY(gf2e::fft_fwd_packed_batch(S.plan, S.FA, S.n, reinterpret_cast<const u32 *>(S.ACC),
                                        2 * S.stride, S.nchunks, 0, na, st));
    GF2E_TRY(gf2e::fft_fwd_packed_batch(S.plan, S.FB, S.n, reinterpret_cast<const u32 *>(S.C),
                                        2 * S.stride, S.nchunks, 0, na, st));
    GF2E_TRY(gf2e::pointwise(S.FA, S.FB, S.n * na, st));
    GF2E_TRY(gf2e::fft_run_batch(S.plan, false, S.FA, S.n, na, st));
    GF2E_TRY(product_tail(S, na, S.C, st));
    GF2E_TRY(gf2e::trin_reduce_batch(S.P, S.pstride, S.ow, 2 * S.r - 1, S.ACC, S.stride, S.r,
                                     S.sdev, na, st));
    // h <- h^(2^m): m squarings of every residue, two per pass, back in H
    return gf2e::frobenius_states(S.H, S.HS, S.stride, na * m, S.r, S.sH, (u64)m, st, 0);
}

int step_kernels(gf2e_scanner &S, int na, cudaStream_t st) {
    return S.m > 1 ? block_kernels(S, na, st) : degree_kernels(S, na, S.F, S.Fs, st);
}

int launch_degree(gf2e_scanner &S, cudaStream_t st) {
    const int na = S.nact;
    if (!S.use_graphs || st != S.own) return step_kernels(S, na, st);
    for (auto &g : S.graphs)
        if (g.first.nact == na && g.first.F == S.F)
            return gf2e::cuda_status(cudaGraphLaunch(g.second, st), "degree graph launch");
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return gf2e::cuda_status(e, "degree graph capture");
    int status = step_kernels(S, na, st);
    e = cudaStreamEndCapture(st, &graph);
    if (status != GF2E_OK) { if (graph) cudaGraphDestroy(graph); return status; }
    if (e != cudaSuccess) return gf2e::cuda_status(e, "degree graph end capture");
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return gf2e::cuda_status(e, "degree graph instantiate");
    if (S.graphs.size() >= 64) {                 // bounded cache
        cudaGraphExecDestroy(S.graphs.front().second);
        S.graphs.erase(S.graphs.begin());
    }
    S.graphs.push_back({gf2e_scanner::GraphKey{na, S.F}, exec});
    return gf2e::cuda_status(cudaGraphLaunch(exec, st), "degree graph launch");
}

// one degree for all resident s, then the interval-end gcds
int degree_step(gf2e_scanner &S, cudaStream_t st) {
    const int na = S.nact;
    GF2E_TRY(launch_degree(S, st));
    const u64 adv = (u64)S.m;                    // degrees per step
    if (S.m == 1) std::swap(S.F, S.Fs);
    S.degree_steps += adv;
    S.sd_pairs += (u64)na * adv;
    std::vector<int> due;
    for (int j = 0; j < na; j++) {
        gf2e_scanner::Slot &sl = S.slot[j];
        sl.k += adv;
        if (sl.k - sl.iv >= sl.L || sl.k >= sl.job.maxd) due.push_back(j);
    }
    if (due.empty()) return GF2E_OK;
    for (size_t q = 0; q < due.size(); q++) {
        int j = due[q];
        S.jobs[q] = gf2e_gcd_job{S.ACC + S.stride * j, S.r, S.T + S.tw * j, S.r + 1,
                                 S.G + S.gcap * q, S.gcap};
    }
    const auto t_gcd = std::chrono::steady_clock::now();
    if (S.r >= GCD_LARGE_BITS) {
        const int par = std::max(1, std::min((int)due.size(), S.gcd_parallel));
        GF2E_TRY(gf2e_gcd_large(S.jobs.data(), (int)due.size(), S.degs.data(), par, nullptr, st));
    } else {
        GF2E_TRY(gf2e_gcd_batch(S.jobs.data(), (int)due.size(), S.degs.data(), S.gws,
                                S.gws_bytes, st));
    }
    S.gcds += due.size();
    S.gcd_seconds +=
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t_gcd).count();
    std::vector<int> retire;
    for (size_t q = 0; q < due.size(); q++) {
        int j = due[q];
        gf2e_scanner::Slot &sl = S.slot[j];
        if (S.degs[q] > 0 || sl.k >= sl.job.maxd) {
            gf2e_scanner::Done D;
            D.tag = sl.job.tag;
            D.res = gf2e_scan_result{sl.job.s, 2, 0, 0, sl.iv + 1, std::min(sl.k, sl.job.maxd)};
            if (S.degs[q] > 0) {
                D.res.status = 3;
                if ((size_t)(S.degs[q] / 64 + 1) <= S.gcap) {
                    cudaError_t e = cudaMemcpyAsync(S.ghost.data(), S.G + S.gcap * q, S.gcap * 8,
                                                    cudaMemcpyDeviceToHost, st);
                    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
                    if (e != cudaSuccess) return gf2e::cuda_status(e, "gcd readback");
                    std::vector<u64> g(S.ghost.begin(), S.ghost.end());
                    u64 d = 0;
                    // the clear intervals (k0, iv] exclude every factor degree
                    // up to iv once iv >= 2 k0: each d <= k0 has a multiple in
                    // (k0, 2 k0], so a factor of degree d would have hit there
                    const u64 clean = sl.iv >= 2 * sl.job.k0 ? sl.iv : 0;
                    if (gf2e::hostpoly::least_factor(g, clean, sl.k, d, D.mask)) {
                        D.res.status = 1;
                        D.res.d = d;
                        D.res.mask_words = D.mask.size();
                        if (d > sl.job.maxd) {       // a block ran past maxd
                            D.res = gf2e_scan_result{sl.job.s, 2, 0, 0, sl.iv + 1, sl.job.maxd};
                            D.mask.clear();
                        }
                    }
                }
            }
            S.done.push_back(std::move(D));
            retire.push_back(j);
        } else {
            sl.iv = sl.k;
            sl.L = gf2e::sched_next(sl.job.sched, (u64)S.m, sl.L, sl.k, sl.job.Lmax);
            GF2E_TRY(gf2e::trin_set_const(S.ACC + S.stride * j, S.stride, 1, S.r, 1, st));
        }
    }
    // refill from the queue, else compact (highest slots first)
    std::sort(retire.begin(), retire.end(), std::greater<int>());
    for (int j : retire) {
        if (!S.queue.empty()) {
            gf2e_scanner::Job job = S.queue.front();
            S.queue.pop_front();
            GF2E_TRY(load_slot(S, j, job, st));
        } else {
            if (j != S.nact - 1) GF2E_TRY(move_slot(S, j, S.nact - 1, st));
            S.nact--;
        }
    }
    return GF2E_OK;
}

}  // namespace

namespace gf2e {
// the scanner's own stream: the serving loop runs independent scanners
// concurrently by stepping each on its own stream
cudaStream_t scanner_stream(gf2e_scanner *S) { return S ? S->own : nullptr; }
}  // namespace gf2e

extern "C" {

int gf2e_scanner_footprint_blocked(uint64_t r, int slots, int block, size_t *bytes) {
    if (!bytes || slots < 1 || r < 5) return gf2e::invalid("bad footprint query");
    if (!(block == 1 || (block >= 2 && block <= 62 && !(block & 1))))
        return gf2e::invalid("scanner: block size must be 1 or even in 2..62");
    Geometry g = geometry(r);
    size_t words = device_words(g, slots, block);
    // gcd workspace: job table + 4 buffers per job (quadratic gcd), or room
    // for 16 members of a half-gcd batch (a batch sizes itself from the
    // memory free when it starts, so more slots only make it run in parts)
    size_t gw = ((size_t)slots * 96 + 255) + (size_t)slots * 4 * (g.tw + 1) * 8;
    if (r >= GCD_LARGE_BITS) {
        int par = 16;
        if (const char *env = getenv("GF2E_SCAN_GCD_PARALLEL")) par = std::max(1, atoi(env));
        gw = (size_t)std::min(par, slots) * HGCD_WORDS_PER_WORD * (g.tw + 1) * 8;
    }
    *bytes = words * 8 + gw;
    return GF2E_OK;
}

int gf2e_scanner_footprint(uint64_t r, int slots, size_t *bytes) {
    return gf2e_scanner_footprint_blocked(r, slots, 1, bytes);
}

int gf2e_scanner_create_blocked(uint64_t r, int slots, int block, gf2e_scanner **out) {
    if (!out || slots < 1 || slots > 4096) return gf2e::invalid("scanner: 1 <= slots <= 4096");
    if (r < 5 || !(r & 1) || r >= (1ull << 31)) return gf2e::invalid("scanner: bad r");
    if (!(block == 1 || (block >= 2 && block <= 62 && !(block & 1))))
        return gf2e::invalid("scanner: block size must be 1 or even in 2..62");
    if ((u64)block >= r) return gf2e::invalid("scanner: block size must be below r");
    Geometry g = geometry(r);
    gf2e_scanner *S = new gf2e_scanner;
    S->r = r;
    S->B = slots;
    S->m = block;
    S->nw = g.nw; S->stride = g.stride; S->tw = g.tw; S->ow = g.ow; S->pstride = g.pstride;
    S->gcap = g.gcap; S->n = g.n; S->nchunks = g.nchunks;
    S->plan = gf2e::cached_plan(g.m);
    if (!S->plan) { delete S; return gf2e::invalid("FFT plan m=%d", g.m); }
    S->wrap = g.wrap;
    S->wm = g.wm;
    if (S->wrap && !gf2e::wrap_mul_plans(S->wm)) {
        delete S;
        return gf2e::invalid("FFT plans for the wrapped product");
    }
    S->dmem_bytes = device_words(g, slots, block) * 8;
    cudaError_t e = cudaMalloc(&S->dmem, S->dmem_bytes);
    if (e != cudaSuccess) { delete S; return gf2e::cuda_status(e, "scanner buffers"); }
    const int B = slots;
    S->F = S->dmem;
    S->Fs = S->F + g.stride * B;
    S->ACC = S->Fs + g.stride * B;
    S->FA = S->ACC + g.stride * B;
    S->FB = S->FA + g.n * B;
    S->P = S->FB + g.n * B;
    S->T = S->P + g.pstride * B;
    S->sdev = S->T + g.tw * B;
    S->G = S->sdev + B;
    if (block > 1) {
        S->H = S->G + g.gcap * B;
        S->HS = S->H + (size_t)block * g.stride * B;
        S->C = S->HS + (size_t)block * g.stride * B;
        S->sH = S->C + g.stride * B;
        S->shH.assign((size_t)block * B, 0);
    }
    if (S->wrap) S->WS = S->dmem + (device_words(g, slots, block) - (size_t)g.wm.per * B);
    std::vector<gf2e_gcd_job> tmp(B, gf2e_gcd_job{S->ACC, r, S->T, r + 1, S->G, g.gcap});
    int st = GF2E_OK;
    if (r < GCD_LARGE_BITS) st = gf2e_gcd_workspace_size(tmp.data(), B, &S->gws_bytes);
    if (st == GF2E_OK && r < GCD_LARGE_BITS) {
        e = cudaMalloc(&S->gws, S->gws_bytes);
        if (e != cudaSuccess) st = gf2e::cuda_status(e, "scanner gcd workspace");
    }
    if (st != GF2E_OK) {
        cudaFree(S->dmem);
        delete S;
        return st;
    }
    e = cudaStreamCreateWithFlags(&S->own, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S->ev_in, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S->ev_out, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        gf2e_scanner_destroy(S);
        return gf2e::cuda_status(e, "scanner stream");
    }
    if (const char *env = getenv("GF2E_SCAN_GRAPHS")) S->use_graphs = env[0] != '0';
    if (const char *env = getenv("GF2E_SCAN_GCD_PARALLEL")) S->gcd_parallel = std::max(1, atoi(env));
    S->slot.resize(B);
    S->shost.assign(B, 0);
    S->thost.assign(g.tw, 0);
    S->ghost.assign(g.gcap, 0);
    S->degs.assign(B, 0);
    S->jobs.resize(B);
    *out = S;
    return GF2E_OK;
}

int gf2e_scanner_create(uint64_t r, int slots, gf2e_scanner **out) {
    return gf2e_scanner_create_blocked(r, slots, 1, out);
}

int gf2e_scanner_destroy(gf2e_scanner *S) {
    if (!S) return GF2E_OK;
    if (S->own) cudaStreamSynchronize(S->own);
    for (auto &g : S->graphs) cudaGraphExecDestroy(g.second);
    if (S->ev_in) cudaEventDestroy(S->ev_in);
    if (S->ev_out) cudaEventDestroy(S->ev_out);
    if (S->own) cudaStreamDestroy(S->own);
    cudaFree(S->gws);
    cudaFree(S->dmem);
    delete S;
    return GF2E_OK;
}

int gf2e_scanner_submit(gf2e_scanner *S, const uint64_t *s_host, int ns, uint64_t k0,
                        uint64_t maxd, uint64_t L0, uint64_t Lmax, uint64_t tag0) {
    if (!S || !s_host || ns < 0) return gf2e::invalid("scanner submit: bad arguments");
    if (!(k0 >= 1 && maxd > k0)) return gf2e::invalid("scanner submit: need 1 <= k0 < maxd");
    for (int i = 0; i < ns; i++)
        if (!(s_host[i] >= 1 && 2 * s_host[i] < S->r))
            return gf2e::invalid("scanner submit: s=%llu outside 1..(r-1)/2",
                                 (unsigned long long)s_host[i]);
    if (Lmax < 1) Lmax = 1;
    if (L0 < 1) L0 = 1;
    if (L0 > Lmax) L0 = Lmax;
    // blocked mode: intervals are whole blocks
    const u64 bm = (u64)S->m;
    L0 = (L0 + bm - 1) / bm * bm;
    Lmax = (Lmax + bm - 1) / bm * bm;
    for (int i = 0; i < ns; i++)
        S->queue.push_back(
            gf2e_scanner::Job{s_host[i], k0, maxd, L0, Lmax, tag0 + (u64)i, S->sched});
    return GF2E_OK;
}

int gf2e_scanner_step(gf2e_scanner *S, int degrees, void *stream) {
    if (!S || degrees < 0) return gf2e::invalid("scanner step: bad arguments");
    // work runs on the scanner's own stream (graphs are captured there),
    // ordered after and before the caller's stream
    cudaStream_t caller = (cudaStream_t)stream;
    cudaError_t e = cudaEventRecord(S->ev_in, caller);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(S->own, S->ev_in, 0);
    if (e != cudaSuccess) return gf2e::cuda_status(e, "scanner stream order");
    int st = fill_slots(*S, S->own);
    const int steps = (degrees + S->m - 1) / S->m;               // blocks in blocked mode
    for (int i = 0; st == GF2E_OK && i < steps && S->nact > 0; i++) st = degree_step(*S, S->own);
    e = cudaEventRecord(S->ev_out, S->own);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(caller, S->ev_out, 0);
    if (st != GF2E_OK) return st;
    return gf2e::cuda_status(e, "scanner stream order");
}

int gf2e_scanner_status(const gf2e_scanner *S, int *queued, int *resident, int *finished,
                        uint64_t *sd_pairs) {
    if (!S) return gf2e::invalid("null scanner");
    if (queued) *queued = (int)S->queue.size();
    if (resident) *resident = S->nact;
    if (finished) *finished = (int)S->done.size();
    if (sd_pairs) *sd_pairs = S->sd_pairs;
    return GF2E_OK;
}

int gf2e_scanner_gcd_time(const gf2e_scanner *S, uint64_t *gcds, double *seconds) {
    if (!S) return gf2e::invalid("null scanner");
    if (gcds) *gcds = S->gcds;
    if (seconds) *seconds = S->gcd_seconds;
    return GF2E_OK;
}

int gf2e_scanner_frontiers(const gf2e_scanner *S, uint64_t *s_host, uint64_t *k_host,
                           uint64_t *tags_host, int cap, int *nout) {
    if (!S || !s_host || !k_host || !nout || cap < 0)
        return gf2e::invalid("scanner frontiers: bad arguments");
    int n = 0;
    for (int j = 0; j < S->nact && n < cap; j++, n++) {
        s_host[n] = S->slot[j].job.s;
        k_host[n] = S->slot[j].iv;
        if (tags_host) tags_host[n] = S->slot[j].job.tag;
    }
    *nout = n;
    return GF2E_OK;
}

int gf2e_scanner_poll(gf2e_scanner *S, gf2e_scan_result *res, uint64_t *tags,
                      uint64_t *masks_host, size_t mask_cap_words, int cap, int *nout) {
    if (!S || !res || !tags || !nout || cap < 0) return gf2e::invalid("scanner poll: bad arguments");
    int k = 0;
    while (k < cap && !S->done.empty()) {
        gf2e_scanner::Done &D = S->done.front();
        res[k] = D.res;
        tags[k] = D.tag;
        if (D.res.status == 1) {
            if (masks_host && D.mask.size() <= mask_cap_words) {
                for (size_t w = 0; w < mask_cap_words; w++)
                    masks_host[(size_t)k * mask_cap_words + w] = w < D.mask.size() ? D.mask[w] : 0;
            } else {
                res[k].status = 3;                     // caller's mask buffer too small
            }
        }
        S->done.pop_front();
        k++;
    }
    *nout = k;
    return GF2E_OK;
}

int gf2e_scanner_set_schedule(gf2e_scanner *S, const gf2e_sched *sched) {
    if (!S) return gf2e::invalid("null scanner");
    GF2E_TRY(gf2e::sched_check(sched));
    S->sched = *sched;
    return GF2E_OK;
}

int gf2e_sched_widths(const gf2e_sched *sched, int block, uint64_t k_start, uint64_t L0,
                      uint64_t Lmax, int n, uint64_t *widths) {
    GF2E_TRY(gf2e::sched_check(sched));
    if (block < 1 || k_start < 2 || n < 0 || (n && !widths))
        return gf2e::invalid("schedule widths: bad arguments");
    const u64 m = (u64)block;
    if (Lmax < 1) Lmax = 1;
    if (L0 < 1) L0 = 1;
    L0 = (std::min(L0, Lmax) + m - 1) / m * m;
    Lmax = (Lmax + m - 1) / m * m;
    u64 w = gf2e::sched_first(*sched, m, k_start, L0), k_end = k_start - 1;
    for (int i = 0; i < n; i++) {
        widths[i] = w;
        k_end += w;
        w = gf2e::sched_next(*sched, m, w, k_end, Lmax);
    }
    return GF2E_OK;
}

int gf2e_scan(uint64_t r, const uint64_t *s_host, int ns, uint64_t k0, uint64_t maxd,
              uint64_t L0, uint64_t Lmax, int batch, gf2e_scan_result *res,
              uint64_t *masks_host, size_t mask_cap_words, void *stream) {
    return gf2e_scan_blocked(r, s_host, ns, k0, maxd, L0, Lmax, batch, 1, res, masks_host,
                             mask_cap_words, stream);
}

int gf2e_scan_blocked(uint64_t r, const uint64_t *s_host, int ns, uint64_t k0, uint64_t maxd,
                      uint64_t L0, uint64_t Lmax, int batch, int block, gf2e_scan_result *res,
                      uint64_t *masks_host, size_t mask_cap_words, void *stream) {
    const gf2e_sched dbl{GF2E_SCHED_DOUBLING, 0, 0, 0.0, 0};
    return gf2e_scan_sched(r, s_host, ns, k0, maxd, &dbl, L0, Lmax, batch, block, res,
                           masks_host, mask_cap_words, stream);
}

int gf2e_scan_sched(uint64_t r, const uint64_t *s_host, int ns, uint64_t k0, uint64_t maxd,
                    const gf2e_sched *sched, uint64_t L0, uint64_t Lmax, int batch, int block,
                    gf2e_scan_result *res, uint64_t *masks_host, size_t mask_cap_words,
                    void *stream) {
    if (!s_host || !res || ns < 1 || batch < 1)
        return gf2e::invalid("gf2e_scan: ns >= 1 and batch >= 1 required");
    GF2E_TRY(gf2e::sched_check(sched));
    gf2e_scanner *S = nullptr;
    GF2E_TRY(gf2e_scanner_create_blocked(r, std::min(batch, ns), block, &S));
    int st = gf2e_scanner_set_schedule(S, sched);
    if (st == GF2E_OK) st = gf2e_scanner_submit(S, s_host, ns, k0, maxd, L0, Lmax, 0);
    std::vector<gf2e_scan_result> tmp(ns);
    std::vector<u64> tags(ns), masks((size_t)ns * mask_cap_words);
    int got = 0;
    while (st == GF2E_OK && got < ns) {
        int q = 0, a = 0;
        st = gf2e_scanner_step(S, 256, stream);
        if (st != GF2E_OK) break;
        gf2e_scanner_status(S, &q, &a, nullptr, nullptr);
        int n = 0;
        st = gf2e_scanner_poll(S, tmp.data() + got, tags.data() + got,
                               masks_host ? masks.data() + (size_t)got * mask_cap_words : nullptr,
                               mask_cap_words, ns - got, &n);
        got += n;
        if (q == 0 && a == 0 && got < ns) { st = gf2e::invalid("scan lost %d results", ns - got); }
    }
    if (st == GF2E_OK) {
        for (int i = 0; i < ns; i++) {
            u64 idx = tags[i];
            res[idx] = tmp[i];
            if (masks_host)
                for (size_t w = 0; w < mask_cap_words; w++)
                    masks_host[idx * mask_cap_words + w] = masks[(size_t)i * mask_cap_words + w];
        }
    }
    gf2e_scanner_destroy(S);
    return st;
}

}  // extern "C"
