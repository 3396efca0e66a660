// tune.cu -- process-wide tuning knobs and the autotuner.
//
// The reference exposes its FFT register-stage depths as runtime knobs read
// from the environment (gf2_cantor_cuda.h:24-60) and tunes them with
// tsfactor's "--bench" autotune (tsfactor.cu:1986-2080): every candidate is
// verified on the device against a reference transform, timed (fwd + inv),
// and the winner is left active and printed as environment settings.  The
// same contract holds here, over this engine's knobs:
//   FFT   tile size (2^11..2^13 elements of shared memory per pass), the
//         least contiguous column count of a tile row, and the number of
//         Taylor / butterfly levels fused per register stage;
//   sieve the strip width of k_strip (entries of best[] per CTA);
//   scan  the gcd interval schedule (L0 doubling to Lmax), from a cost
//         model over measured per-degree and per-gcd costs, and the block
//         size of the blocked DDF from the measured modmul and squaring costs.
#include "gf2e_internal.cuh"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

namespace gf2e {
int fft_plan_create_cfg(int m, const gf2e_tune &cfg, gf2e_fft_plan **out);
int fft_run(const gf2e_fft_plan *plan, bool forward, u64 *f, cudaStream_t st);
}  // namespace gf2e

namespace {

std::mutex g_tune_mu;
bool g_tune_init = false;
gf2e_tune g_tune;

gf2e_tune builtin_default() {
    gf2e_tune t;
    t.fft_tile_log = 0;              // 0: by transform size (the autotuned B200 choices)
    t.fft_cmin = 0;
    t.fft_taylor_lv = 3;
    t.fft_bfly_lv = 3;
    t.sieve_strip_log = 12;
    return t;
}

bool pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }

const char *tune_problem(const gf2e_tune &t) {
    if (t.fft_tile_log != 0 && (t.fft_tile_log < 11 || t.fft_tile_log > 13))
        return "fft_tile_log not 0 (by size) or 11..13";
    if (t.fft_cmin != 0 && (!pow2(t.fft_cmin) || t.fft_cmin > 16))
        return "fft_cmin not 0 (by size) or one of 1, 2, 4, 8, 16";
    if (t.fft_taylor_lv < 1 || t.fft_taylor_lv > 3) return "fft_taylor_lv outside 1..3";
    if (t.fft_bfly_lv < 1 || t.fft_bfly_lv > 3) return "fft_bfly_lv outside 1..3";
    if (t.sieve_strip_log < 10 || t.sieve_strip_log > 14) return "sieve_strip_log outside 10..14";
    return nullptr;
}

void env_int(const char *name, int *dst) {
    const char *e = getenv(name);
    if (e && *e) *dst = atoi(e);
}

// caller holds g_tune_mu
void ensure_init() {
    if (g_tune_init) return;
    gf2e_tune t = builtin_default();
    env_int("GF2E_FFT_TILE_LOG", &t.fft_tile_log);
    env_int("GF2E_FFT_CMIN", &t.fft_cmin);
    env_int("GF2E_FFT_TAYLOR_LV", &t.fft_taylor_lv);
    env_int("GF2E_FFT_BFLY_LV", &t.fft_bfly_lv);
    env_int("GF2E_SIEVE_STRIP_LOG", &t.sieve_strip_log);
    if (tune_problem(t)) {
        fprintf(stderr, "gf2e: ignoring GF2E_* tuning environment (%s)\n", tune_problem(t));
        t = builtin_default();
    }
    g_tune = t;
    g_tune_init = true;
}

__global__ void k_count_diff(const u64 *__restrict__ a, const u64 *__restrict__ b, u64 n,
                             unsigned long long *__restrict__ cnt) {
    unsigned long long c = 0;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (u64)gridDim.x * blockDim.x)
        c += (a[i] != b[i]);
    for (int o = 16; o; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(cnt, c);
}

// number of differing words (synchronises the stream)
int count_diff(const u64 *a, const u64 *b, u64 n, unsigned long long *d_cnt, cudaStream_t st,
               unsigned long long *out) {
    cudaError_t e = cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return gf2e::cuda_status(e, "diff reset");
    k_count_diff<<<gf2e::grid_for(n, 256), 256, 0, st>>>(a, b, n, d_cnt);
    GF2E_CHECK_LAUNCH("k_count_diff");
    e = cudaMemcpyAsync(out, d_cnt, sizeof *out, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return gf2e::cuda_status(e, "diff read");
}

void report_line(std::string &rep, const char *fmt, ...) {
    char buf[256];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    rep += buf;
}

void report_out(const std::string &rep, char *report, size_t cap) {
    if (!report || !cap) return;
    size_t n = std::min(cap - 1, rep.size());
    memcpy(report, rep.data(), n);
    report[n] = 0;
}

u64 splitmix(u64 &st) {
    u64 z = (st += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// device buffers released on every return path
struct DevBufs {
    std::vector<void *> p;
    ~DevBufs() {
        for (void *q : p) cudaFree(q);
    }
    int alloc(void **dst, size_t bytes) {
        cudaError_t e = cudaMalloc(dst, bytes);
        if (e != cudaSuccess) return gf2e::cuda_status(e, "autotune buffer");
        p.push_back(*dst);
        return GF2E_OK;
    }
};

struct StreamEvents {
    cudaStream_t st = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    ~StreamEvents() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
        if (st) cudaStreamDestroy(st);
    }
    int init() {
        cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreate(&a);
        if (e == cudaSuccess) e = cudaEventCreate(&b);
        return gf2e::cuda_status(e, "autotune stream");
    }
};

}  // namespace

namespace gf2e {

gf2e_tune tune_current() {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    ensure_init();
    return g_tune;
}

}  // namespace gf2e

extern "C" {

int gf2e_tune_default(gf2e_tune *t) {
    if (!t) return gf2e::invalid("null tune");
    *t = builtin_default();
    return GF2E_OK;
}

int gf2e_tune_get(gf2e_tune *t) {
    if (!t) return gf2e::invalid("null tune");
    *t = gf2e::tune_current();
    return GF2E_OK;
}

int gf2e_tune_set(const gf2e_tune *t) {
    if (!t) return gf2e::invalid("null tune");
    if (const char *why = tune_problem(*t)) return gf2e::invalid("gf2e_tune_set: %s", why);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune = *t;
    g_tune_init = true;
    return GF2E_OK;
}

int gf2e_fft_autotune(int m, int reps, gf2e_tune *best, double *best_ms, char *report,
                      size_t report_cap) {
    if (m < 4 || m > 28) return gf2e::invalid("gf2e_fft_autotune: m=%d outside 4..28", m);
    if (reps < 1) reps = 1;
    const u64 n = (u64)1 << m;
    const gf2e_tune base = gf2e::tune_current();
    DevBufs bufs;
    u64 *d_in, *d_ref, *d_w;
    unsigned long long *d_cnt;
    GF2E_TRY(bufs.alloc((void **)&d_in, n * 8));
    GF2E_TRY(bufs.alloc((void **)&d_ref, n * 8));
    GF2E_TRY(bufs.alloc((void **)&d_w, n * 8));
    GF2E_TRY(bufs.alloc((void **)&d_cnt, 8));
    StreamEvents se;
    GF2E_TRY(se.init());
    {
        std::vector<u64> h(n);
        u64 s = 0xfeedfaceull;
        for (auto &w : h) w = splitmix(s);
        cudaError_t e = cudaMemcpy(d_in, h.data(), n * 8, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return gf2e::cuda_status(e, "autotune input");
    }
    // reference forward transform under the built-in default tuning
    {
        gf2e_fft_plan *p = nullptr;
        GF2E_TRY(gf2e::fft_plan_create_cfg(m, builtin_default(), &p));
        cudaError_t e = cudaMemcpyAsync(d_ref, d_in, n * 8, cudaMemcpyDeviceToDevice, se.st);
        int st = (e == cudaSuccess) ? gf2e::fft_run(p, true, d_ref, se.st)
                                    : gf2e::cuda_status(e, "autotune copy");
        if (st == GF2E_OK) st = gf2e::cuda_status(cudaStreamSynchronize(se.st), "autotune ref");
        gf2e_fft_plan_destroy(p);
        GF2E_TRY(st);
    }
    std::string rep;
    gf2e_tune win = base;
    double win_ms = 1e30;
    bool have = false;
    for (int tl = 11; tl <= 13; tl++)
        for (int cmin : {2, 4, 8, 16})
            for (int tlv = 1; tlv <= 3; tlv++)
                for (int blv = 1; blv <= 3; blv++) {
                    gf2e_tune c = base;
                    c.fft_tile_log = tl;
                    c.fft_cmin = cmin;
                    c.fft_taylor_lv = tlv;
                    c.fft_bfly_lv = blv;
                    gf2e_fft_plan *p = nullptr;
                    GF2E_TRY(gf2e::fft_plan_create_cfg(m, c, &p));
                    unsigned long long dfw = 1, dinv = 1;
                    float ms = 0;
                    cudaError_t e = cudaMemcpyAsync(d_w, d_in, n * 8, cudaMemcpyDeviceToDevice, se.st);
                    int st = (e == cudaSuccess) ? gf2e::fft_run(p, true, d_w, se.st)
                                                : gf2e::cuda_status(e, "autotune copy");
                    if (st == GF2E_OK) st = count_diff(d_w, d_ref, n, d_cnt, se.st, &dfw);
                    if (st == GF2E_OK) st = gf2e::fft_run(p, false, d_w, se.st);
                    if (st == GF2E_OK) st = count_diff(d_w, d_in, n, d_cnt, se.st, &dinv);
                    // timing: one warm-up fwd+inv, then reps of fwd+inv
                    if (st == GF2E_OK && dfw == 0 && dinv == 0) {
                        st = gf2e::fft_run(p, true, d_w, se.st);
                        if (st == GF2E_OK) st = gf2e::fft_run(p, false, d_w, se.st);
                        if (st == GF2E_OK) cudaEventRecord(se.a, se.st);
                        for (int r = 0; r < reps && st == GF2E_OK; r++) {
                            st = gf2e::fft_run(p, true, d_w, se.st);
                            if (st == GF2E_OK) st = gf2e::fft_run(p, false, d_w, se.st);
                        }
                        if (st == GF2E_OK) {
                            cudaEventRecord(se.b, se.st);
                            e = cudaEventSynchronize(se.b);
                            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, se.a, se.b);
                            st = gf2e::cuda_status(e, "autotune timing");
                            ms /= reps;
                        }
                    }
                    gf2e_fft_plan_destroy(p);
                    GF2E_TRY(st);
                    const bool ok = (dfw == 0 && dinv == 0);
                    report_line(rep, "%d %d %d %d %.4f %s\n", tl, cmin, tlv, blv, ok ? ms : -1.0,
                                ok ? "ok" : "MISMATCH");
                    if (ok && ms < win_ms) { win = c; win_ms = ms; have = true; }
                }
    report_out(rep, report, report_cap);
    if (!have) {
        gf2e::set_error("gf2e_fft_autotune: no candidate matched the reference transform");
        return GF2E_ERR_INTERNAL;
    }
    GF2E_TRY(gf2e_tune_set(&win));
    if (best) *best = win;
    if (best_ms) *best_ms = win_ms;
    return GF2E_OK;
}

int gf2e_sieve_autotune(uint64_t r, int dmax, uint64_t smax, int reps, gf2e_tune *best,
                        double *best_ms, char *report, size_t report_cap) {
    if (reps < 1) reps = 1;
    size_t ws_bytes = 0;
    GF2E_TRY(gf2e_sieve_workspace_size(dmax, &ws_bytes));
    DevBufs bufs;
    void *ws;
    u64 *d_ref, *d_b;
    unsigned long long *d_cnt;
    GF2E_TRY(bufs.alloc(&ws, ws_bytes));
    GF2E_TRY(bufs.alloc((void **)&d_ref, 8 * (smax + 1)));
    GF2E_TRY(bufs.alloc((void **)&d_b, 8 * (smax + 1)));
    GF2E_TRY(bufs.alloc((void **)&d_cnt, 8));
    StreamEvents se;
    GF2E_TRY(se.init());
    const gf2e_tune base = gf2e::tune_current();
    std::string rep;
    gf2e_tune win = base;
    double win_ms = 1e30;
    bool have = false;
    int st = GF2E_OK;
    for (int pass = 0; pass < 2 && st == GF2E_OK; pass++) {
        // pass 0: reference result with the built-in strip width
        for (int sl = 10; sl <= 14 && st == GF2E_OK; sl++) {
            if (pass == 0 && sl != builtin_default().sieve_strip_log) continue;
            gf2e_tune c = base;
            c.sieve_strip_log = sl;
            st = gf2e_tune_set(&c);
            if (st != GF2E_OK) break;
            u64 *dst = pass == 0 ? d_ref : d_b;
            float ms = 0;
            const int nrun = pass == 0 ? 1 : reps + 1;
            for (int rr = 0; rr < nrun && st == GF2E_OK; rr++) {    // rr = 0 is warm-up
                if (rr == 1) cudaEventRecord(se.a, se.st);
                st = gf2e_sieve_fill(dst, smax, se.st);
                if (st == GF2E_OK) st = gf2e_sieve_run(r, 2, dmax, smax, dst, ws, ws_bytes, se.st);
            }
            if (st != GF2E_OK) {
                // a strip width whose progression list overflows is skipped
                if (st == GF2E_ERR_OVERFLOW && pass == 1) {
                    report_line(rep, "%d -1 OVERFLOW\n", sl);
                    st = GF2E_OK;
                    continue;
                }
                break;
            }
            if (pass == 0) {                  // reference result only, not timed
                st = gf2e::cuda_status(cudaStreamSynchronize(se.st), "sieve autotune reference");
                continue;
            }
            cudaEventRecord(se.b, se.st);
            cudaError_t e = cudaEventSynchronize(se.b);
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, se.a, se.b);
            st = gf2e::cuda_status(e, "sieve autotune timing");
            if (st != GF2E_OK) break;
            ms /= reps;
            unsigned long long diff = 1;
            st = count_diff(d_b, d_ref, smax + 1, d_cnt, se.st, &diff);
            if (st != GF2E_OK) break;
            report_line(rep, "%d %.4f %s\n", sl, diff ? -1.0 : ms, diff ? "MISMATCH" : "ok");
            if (!diff && ms < win_ms) { win = c; win_ms = ms; have = true; }
        }
    }
    report_out(rep, report, report_cap);
    if (st != GF2E_OK) {
        gf2e_tune_set(&base);
        return st;
    }
    if (!have) {
        gf2e_tune_set(&base);
        gf2e::set_error("gf2e_sieve_autotune: no strip width matched the reference sieve");
        return GF2E_ERR_INTERNAL;
    }
    GF2E_TRY(gf2e_tune_set(&win));
    if (best) *best = win;
    if (best_ms) *best_ms = win_ms;
    return GF2E_OK;
}

int gf2e_scan_choose_block(double t_mul, double t_sq, int *block) {
    if (!block || !(t_mul > 0) || !(t_sq > 0)) return gf2e::invalid("gf2e_scan_choose_block: bad arguments");
    // per degree: m squarings of the m h's... m * t_sq + t_mul / m, least at
    // m = sqrt(t_mul / t_sq) (tsfactor.cu:1979-1984 picks the same balance)
    double m = std::sqrt(t_mul / t_sq);
    int mi = 2 * (int)std::lround(m / 2.0);
    if (mi < 2) mi = 2;
    if (mi > 62) mi = 62;
    *block = mi;
    return GF2E_OK;
}

int gf2e_scan_choose_interval(uint64_t k0, uint64_t maxd, double t_degree, double t_gcd,
                              uint64_t *L0_out, uint64_t *Lmax_out, double *expected_cost) {
    if (!L0_out || !Lmax_out || k0 < 1 || maxd <= k0 || !(t_degree > 0) || !(t_gcd >= 0))
        return gf2e::invalid("gf2e_scan_choose_interval: bad arguments");
    // P(least factor degree > D) = min(1, k0 / D) for a survivor of a k0-deep
    // sieve; a gcd is paid at the end of every interval reached
    auto cost = [&](u64 L0, u64 Lmax) {
        double c = 0;
        u64 lo = k0, L = L0;
        while (lo < maxd) {
            u64 hi = std::min<u64>(maxd, lo + L);
            double p_alive = (double)k0 / (double)lo;     // lo >= k0
            c += p_alive * ((double)(hi - lo) * t_degree + t_gcd);
            lo = hi;
            L = std::min<u64>(2 * L, Lmax);
        }
        return c;
    };
    double best_c = 1e300;
    u64 bL0 = 64, bLmax = 4096;
    for (u64 L0 = 1; L0 <= (1ull << 20); L0 <<= 1)
        for (u64 Lmax = L0; Lmax <= (1ull << 22); Lmax <<= 1) {
            double c = cost(L0, Lmax);
            if (c < best_c * (1 - 1e-12)) { best_c = c; bL0 = L0; bLmax = Lmax; }
        }
    *L0_out = bL0;
    *Lmax_out = bLmax;
    if (expected_cost) *expected_cost = best_c;
    return GF2E_OK;
}

}  // extern "C"
