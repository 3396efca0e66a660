/*
 * gf2e.h -- C ABI of the B200 engine for smallest irreducible factors of
 * x^r + x^s + 1 over GF(2) (libgf2e.so).
 *
 * Plain pointers and sizes only.  Every entry point returns an int status
 * (GF2E_OK = 0, negative on error) and never exits the process; the C++
 * drop-in headers (gf2e_cantor.hpp, gf2e_trinomial.hpp) turn a non-zero
 * status into the reference's print-and-exit behaviour.  Pointers named
 * *_dev are device pointers; `stream` is a cudaStream_t (NULL = legacy
 * default stream).  All launches are asynchronous on `stream` unless noted.
 *
 * Bit layout (shared with the reference, gf2_gcd.h:1-4): little-endian
 * uint64 words, bit i of word w is the coefficient of x^(64w+i); a residue
 * mod x^r + x^s + 1 has nw = ceil(r/64) words and bits >= r are zero.
 *
 * Each declaration names the reference interface it replaces.
 */
#ifndef GF2E_H
#define GF2E_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GF2E_ABI_VERSION 1

/* status codes */
#define GF2E_OK 0
#define GF2E_ERR_INVALID -1        /* bad argument (the reference exit(1)s) */
#define GF2E_ERR_CUDA -2           /* CUDA runtime error, see gf2e_last_error() */
#define GF2E_ERR_NOMEM -3          /* workspace too small / allocation failed */
#define GF2E_ERR_UNSUPPORTED_R -4  /* gcd(r, 2^d - 1) != 1 (sieve_ref.cpp:79-83) */
#define GF2E_ERR_TIMEOUT -5        /* a bounded device-side wait gave up */
#define GF2E_ERR_OVERFLOW -6       /* a fixed-capacity device queue overflowed */
#define GF2E_ERR_INTERNAL -7       /* consistency check failed on the device */

int gf2e_abi_version(void);
const char *gf2e_status_string(int status);
/* Human-readable detail of the last error raised on the calling thread. */
const char *gf2e_last_error(void);
/* Synchronize `stream` and return GF2E_ERR_CUDA if any launch failed. */
int gf2e_stream_sync(void *stream);

/* Device memory helpers for callers without their own allocator (the
 * reference's contexts cudaMalloc in init, gf2_trinomial_cuda.h:100-116).
 * The copies are ordered on `stream` and return after it has drained. */
int gf2e_device_alloc(void **ptr_dev, size_t bytes);
int gf2e_device_free(void *ptr_dev);
int gf2e_copy_to_host(void *dst_host, const void *src_dev, size_t bytes, void *stream);
int gf2e_copy_to_device(void *dst_dev, const void *src_host, size_t bytes, void *stream);

/* ======================================================================
 * (a) Zech-log sieve.
 * Replaces coarse_sieve.cu run_gpu (1119-1225) / sieve_degree_gpu (852-918)
 * and sieve_ref.cpp run_sieve (125-134).  best_dev[s], s = 0..smax, holds
 * the packed key (d << 48) | mask of the smallest-degree, then numerically
 * least, irreducible factor p of x^r + x^s + 1 with dmin <= d <= dmax; all
 * ones where none was found.  Keys are merged with min, so degrees may be
 * sieved in any order and a preloaded best[] (coarse_sieve --load) is
 * extended exactly.
 * ====================================================================== */

/* Device workspace bytes for gf2e_sieve_run up to degree dmax (<= 40). */
int gf2e_sieve_workspace_size(int dmax, size_t *bytes);

/* best_dev[0..smax] = UINT64_MAX (coarse_sieve.cu k_fill 301-305). */
int gf2e_sieve_fill(uint64_t *best_dev, uint64_t smax, void *stream);

/* Sieve degrees dmin..dmax (2 <= dmin <= dmax <= 40) into best_dev.
 * Degrees <= 31 use dense antilog/log tables of 2^d entries (2 x 8 GB at
 * d = 31).  Degrees 32..40 keep 64-bit field elements and store only the log
 * table, in value slices as large as the workspace allows (the reference's
 * wide-field low-memory mode, coarse_sieve.cu:920-1117): each slice costs
 * one walk over the 2^d - 1 exponents and one pass over the coset leaders.
 * Any workspace of at least the dense tables (when dmin <= 31) and 256 MB
 * (when dmax >= 32) works; gf2e_sieve_workspace_size gives one slice up to
 * 64 GB (GF2E_SIEVE_WIDE_GB overrides).
 * Host-side per-degree setup (primitive polynomial search) is cached.
 * Returns GF2E_ERR_UNSUPPORTED_R when gcd(r mod (2^d-1), 2^d-1) != 1 for
 * some d in range, before launching anything.  All degrees are enqueued on
 * `stream`; the call then reads a small status block, so it returns after
 * the sieve has finished on the device. */
int gf2e_sieve_run(uint64_t r, int dmin, int dmax, uint64_t smax,
                   uint64_t *best_dev, void *workspace_dev,
                   size_t workspace_bytes, void *stream);

/* Read back per-degree statistics of the last gf2e_sieve_run on this
 * workspace (sized for `dmax`): coset classes and marks, arrays of dmax + 1
 * entries indexed by d (sieve_ref.cpp:128-132 prints the same counts).
 * Synchronizes `stream`. */
int gf2e_sieve_stats(const void *workspace_dev, int dmax, uint64_t *classes_host,
                     uint64_t *marks_host, void *stream);

/* Smallest primitive polynomial of degree d, 2 <= d <= 40
 * (gf2_field_setup.h:49-58, gf2_wide_setup.h:44-53).  Host only. */
uint64_t gf2e_primitive_poly(int d);

/* ======================================================================
 * (b) Squaring with trinomial fold reduction in GF(2)[x]/(x^r + x^s + 1).
 * Requires r odd, 1 <= s, 2s < r (gf2_trinomial_cuda.h:118-123).
 * ====================================================================== */

/* out = in^2 mod T, single pass (tsfactor.cu k_square_fused 139-186;
 * gf2_trinomial_cuda.h TrinGPU::square_A 149-154).  in != out. */
int gf2e_trin_square(const uint64_t *in_dev, uint64_t *out_dev, uint64_t r,
                     uint64_t s, void *stream);

/* Batched repeated squaring: each of `nstates` states (state i at
 * states_dev + i*stride_words, stride_words >= nw, even) is squared k times
 * mod x^r + x^(s_i) + 1, s_i = s_dev[i] (device array).  scratch_dev has the
 * same shape as states_dev; the result is left in states_dev.  Two squarings
 * run per pass over the states (F -> F^4 mod T) where r < 2^31; the word
 * after an odd nw in each stride is padding and may be overwritten.
 * (trinomial_stage2.cu run loop 232-253: F_k = x^(2^k) mod T, many s at once.) */
int gf2e_trin_square_batch(uint64_t *states_dev, uint64_t *scratch_dev,
                           size_t stride_words, int nstates, uint64_t r,
                           const uint64_t *s_dev, uint32_t k, void *stream);

/* Squarings per pass that gf2e_trin_square_batch uses for this r, stride
 * and state count: 2, or 1 where the fused pass does not apply or does not
 * pay (r >= 2^31 - 2^16, an odd stride, states and scratch small enough to
 * stay in L2 (at most 96 MB), or GF2E_SQUARINGS_PER_PASS=1 in the
 * environment; GF2E_SQUARINGS_PER_PASS=2 uses the fused pass wherever it
 * applies).  Host only. */
int gf2e_trin_squarings_per_pass(uint64_t r, size_t stride_words, int nstates);

/* Host-buffer form of the above, the whole of trinomial_stage2.cu `run`
 * (195-277) for many s with k0 > k1: F_k = x^(2^k) mod x^r + x^(s_i) + 1 for
 * every s_host[i], written to out_host + i*out_stride_words (nw words each).
 * Device memory is a per-thread workspace kept between calls; returns after
 * the results are in host memory. */
int gf2e_trin_frobenius_host(uint64_t r, const uint64_t *s_host, int nstates,
                             uint32_t k, uint64_t *out_host,
                             size_t out_stride_words, void *stream);

/* states <- x (gf2_trinomial_cuda.h k_set_x 80-84), nstates at stride. */
int gf2e_trin_set_x(uint64_t *states_dev, size_t stride_words, int nstates,
                    uint64_t r, void *stream);

/* states <- 1 (TrinGPU::reset_acc 124-128; tsfactor.cu k_set_one 198-202). */
int gf2e_trin_set_one(uint64_t *states_dev, size_t stride_words, int nstates,
                      uint64_t r, void *stream);

/* out (nw words) = prod mod T where prod has prod_bits <= 2r - 1 bits,
 * stored in ceil(prod_bits/64) words (TrinGPU::reduce 136-146). */
int gf2e_trin_reduce(const uint64_t *prod_dev, uint64_t prod_bits,
                     uint64_t *out_dev, uint64_t r, uint64_t s, void *stream);

/* ======================================================================
 * (c) Cantor additive FFT over GF(2^64) and GF(2)[x] multiplication.
 * Replaces gf2_cantor_cuda.h CudaFFT (361-521) and gf2_cantor_engine.h
 * gf2x_fft_mul_buf / gf2x_fft_mul (207-242).  Transform points and order
 * are the reference's: values f(W-indexed points) in natural order.
 * ====================================================================== */
typedef struct gf2e_fft_plan gf2e_fft_plan;

/* The Cantor basis b[0..len) (CantorBasis::build, gf2_cantor_engine.h:78-103). */
int gf2e_cantor_basis(uint64_t *basis64, int *len);

/* Plan for transforms of n = 2^m points, 1 <= m <= 30 (CudaFFT::init). */
int gf2e_fft_plan_create(int m, gf2e_fft_plan **plan);
int gf2e_fft_plan_destroy(gf2e_fft_plan *plan);
int gf2e_fft_plan_m(const gf2e_fft_plan *plan);
/* Tile passes of the forward and inverse transform (each reads and writes
 * the n points once): the memory traffic a transform of this plan needs. */
int gf2e_fft_plan_passes(const gf2e_fft_plan *plan, int *fwd, int *inv);

/* In-place forward / inverse transform of n device words (CudaFFT::fwd/inv). */
int gf2e_fft_fwd(const gf2e_fft_plan *plan, uint64_t *f_dev, void *stream);
int gf2e_fft_inv(const gf2e_fft_plan *plan, uint64_t *f_dev, void *stream);

/* Twiddle table W[t], t < n/2 (CudaFFT::dW / CantorFFT::W), to host memory. */
int gf2e_fft_twiddles(const gf2e_fft_plan *plan, uint64_t *W_host);

/* The product's element-wise steps on device buffers, as the reference's
 * kernels (gf2_cantor_cuda.h:114-156):
 *   pack:        f[k] = 32-bit chunk k of a (nwords words) for k < nchunks,
 *                0 for nchunks <= k < n (k_pack);
 *   pointwise:   fa[k] = fa[k] * fb[k] in GF(2^64), k < n (k_pointwise);
 *   overlap_add: out[w] = XOR of the 64-bit coefficients f[k], k < nchunks,
 *                placed at bit 32 k, for w < owords (k_overlap_add). */
int gf2e_fft_pack(const uint64_t *a_dev, size_t nwords, uint64_t *f_dev,
                  size_t nchunks, size_t n, void *stream);
int gf2e_fft_pointwise(uint64_t *fa_dev, const uint64_t *fb_dev, size_t n,
                       void *stream);
int gf2e_fft_overlap_add(const uint64_t *f_dev, size_t nchunks, uint64_t *out_dev,
                         size_t owords, void *stream);

/* FFT size exponent for an abits x bbits product (gf2_cantor_engine.h:232-238)
 * and the product's word count (mul_out_words, :201-203). */
int gf2e_mul_fft_m(uint64_t abits, uint64_t bbits);
size_t gf2e_mul_out_words(uint64_t abits, uint64_t bbits);

/* out = a * b over GF(2)[x] (gf2x_fft_mul_buf).  All device pointers; plan
 * size must be >= gf2e_mul_fft_m(abits, bbits); fa, fb: 2^m words each of
 * scratch; out has gf2e_mul_out_words(abits, bbits) words, fully written. */
int gf2e_mul(const gf2e_fft_plan *plan, const uint64_t *a_dev, uint64_t abits,
             const uint64_t *b_dev, uint64_t bbits, uint64_t *out_dev,
             uint64_t *fa_dev, uint64_t *fb_dev, void *stream);

/* The same product with no memory allocated by the call: no counterpart in
 * the reference.  For callers that cannot allocate device memory while they
 * run (an HBM budget fixed at start-up, or a loop that must not let an
 * allocator call synchronise the device).  The transform scratch and
 * twiddle tables are fixed arrays inside the library, sized for transforms
 * of at most 2^GF2E_MUL_NOALLOC_MAX_M points, i.e.
 * ceil(abits/32) + ceil(bbits/32) - 1 <= 2^18; larger products return
 * GF2E_ERR_INVALID.  Every GPU that loads the library holds the 4 MiB of
 * scratch until the process exits.  The first call on a device sets up that
 * device (symbol addresses, twiddle upload, pass schedules) and should come
 * before any stream capture.  All calls share the scratch, which keeps the
 * last call's contents (nothing is read from it before being written): calls
 * that overlap on the GPU, e.g. on two streams, race.  a_dev, b_dev and
 * out_dev (gf2e_mul_out_words words) are the caller's device buffers.  Calls
 * after a cudaDeviceReset in the same process are not supported (the reset
 * drops the uploaded tables the set-up left on the device). */
#define GF2E_MUL_NOALLOC_MAX_M 18
int gf2e_mul_noalloc(const uint64_t *a_dev, uint64_t abits, const uint64_t *b_dev,
                     uint64_t bbits, uint64_t *out_dev, void *stream);

/* One product in a batch (config: many uneven products in one call). */
typedef struct gf2e_mul_job {
    const uint64_t *a_dev;
    uint64_t abits;
    const uint64_t *b_dev;
    uint64_t bbits;
    uint64_t *out_dev;      /* gf2e_mul_out_words(abits, bbits) words */
} gf2e_mul_job;

/* Scratch bytes gf2e_mul_batch needs for these jobs. */
int gf2e_mul_batch_workspace_size(const gf2e_mul_job *jobs_host, int njobs,
                                  size_t *bytes);

/* All products of jobs_host[0..njobs) on the device; plans are created and
 * cached per FFT size inside the library. */
int gf2e_mul_batch(const gf2e_mul_job *jobs_host, int njobs, void *workspace_dev,
                   size_t workspace_bytes, void *stream);

/* ======================================================================
 * (d) gcd over GF(2)[x], batched, one GPU thread block per pair.
 * Replaces the CPU gcd of the interval accumulator (trinomial_scan.cu:64-141
 * GcdPool; gf2_gcd.h:48-75 poly_gcd_naive, same return convention: deg(gcd),
 * 0 for gcd = 1 and for gcd(0, 0)).
 * ====================================================================== */
typedef struct gf2e_gcd_job {
    const uint64_t *a_dev;   /* operands, ceil(bits/64) words, not modified */
    uint64_t abits;
    const uint64_t *b_dev;
    uint64_t bbits;
    uint64_t *g_dev;         /* receives the gcd if it fits g_cap_words (or NULL) */
    size_t g_cap_words;
} gf2e_gcd_job;

int gf2e_gcd_workspace_size(const gf2e_gcd_job *jobs_host, int njobs, size_t *bytes);
/* deg_host[i] = deg gcd(a_i, b_i).  Returns after the results are on the host;
 * GF2E_ERR_TIMEOUT if a job exceeded its round bound (cannot happen for
 * valid inputs; reported instead of looping). */
int gf2e_gcd_batch(const gf2e_gcd_job *jobs_host, int njobs, int64_t *deg_host,
                   void *workspace_dev, size_t workspace_bytes, void *stream);

/* ======================================================================
 * (e) Deep scan of sieve survivors (trinomial_scan.cu:240-381 scan_one_s,
 * 542-697 main), batched over the s values on one GPU.
 * ====================================================================== */
typedef struct gf2e_scan_result {
    uint64_t s;
    int status;           /* 1: least factor found (d, mask); 2: none of degree
                             <= maxd ("s u"); 3: a factor with degree in
                             [rlo, rhi] that could not be isolated ("s rA-B") */
    uint64_t d;           /* least factor degree (status 1) */
    uint64_t mask_words;  /* words of the factor written to the mask buffer */
    uint64_t rlo, rhi;    /* interval of the hit */
} gf2e_scan_result;

/* Least-degree irreducible factor of x^r + x^s + 1 with degree in (k0, maxd]
 * for every s_host[i] (sieve survivors: no factor of degree <= k0), and the
 * numerically least factor of that degree, written to
 * masks_host + i*mask_cap_words.  Intervals of L0, 2*L0, ... <= Lmax degrees
 * between gcd checks (trinomial_scan --l0/--interval).  `batch` s values are
 * resident on the device at once; retired s are replaced from the list.
 * Returns after all results are on the host. */
int gf2e_scan(uint64_t r, const uint64_t *s_host, int ns, uint64_t k0, uint64_t maxd,
              uint64_t L0, uint64_t Lmax, int batch, gf2e_scan_result *results_host,
              uint64_t *masks_host, size_t mask_cap_words, void *stream);

/* gf2e_scan with the multi-level blocking DDF of the reference's tsfactor
 * (tsfactor.cu:1-27, k_horner_fused/k_mulx_xor 71-126, do_block 999-1019):
 * block = m even in 2..62 degrees per step (1 = gf2e_scan): per s the m
 * elementary symmetric functions of the block's Frobenius iterates stay on
 * the device, each block costs one Horner pass, one modmul and m*m
 * squarings.  Intervals are rounded up to whole blocks; results are those
 * of gf2e_scan (a factor found past maxd in the last block reports "u"). */
int gf2e_scan_blocked(uint64_t r, const uint64_t *s_host, int ns, uint64_t k0, uint64_t maxd,
                      uint64_t L0, uint64_t Lmax, int batch, int block,
                      gf2e_scan_result *results_host, uint64_t *masks_host,
                      size_t mask_cap_words, void *stream);

/* Interval schedules: the cadence of interval gcds (results do not depend
 * on it, only the cost does).
 *   GF2E_SCHED_DOUBLING  L0, 2 L0, 4 L0, ... capped at Lmax degrees
 *                        (trinomial_scan --l0/--interval; the default)
 *   GF2E_SCHED_LINEAR    q0, 2 q0, 3 q0, ... blocks (tsfactor's QSched,
 *                        tsfactor.cu:831-858, --q0)
 *   GF2E_SCHED_OPT       tsfactor's Euler-optimal widths for a gcd that
 *                        costs G degrees of scanning, geometric floor rho
 *                        (tsfactor.cu:837-891, --sched opt --sched-G
 *                        --sched-rho; the reference's defaults are G = 4000,
 *                        rho = 1.25)
 * qcap > 0 caps LINEAR and OPT intervals at qcap blocks (tsfactor --Zq). */
enum { GF2E_SCHED_DOUBLING = 0, GF2E_SCHED_LINEAR = 1, GF2E_SCHED_OPT = 2 };
typedef struct gf2e_sched {
    int mode;
    uint64_t q0;
    uint64_t G;
    double rho;
    uint64_t qcap;
} gf2e_sched;

/* The first n interval widths (degrees) of a scan whose first interval
 * starts at degree k_start >= 2 with `block` degrees per block. */
int gf2e_sched_widths(const gf2e_sched *sched, int block, uint64_t k_start, uint64_t L0,
                      uint64_t Lmax, int n, uint64_t *widths_host);

/* gf2e_scan_blocked under an interval schedule (L0 and Lmax are read by
 * GF2E_SCHED_DOUBLING only). */
int gf2e_scan_sched(uint64_t r, const uint64_t *s_host, int ns, uint64_t k0, uint64_t maxd,
                    const gf2e_sched *sched, uint64_t L0, uint64_t Lmax, int batch, int block,
                    gf2e_scan_result *results_host, uint64_t *masks_host,
                    size_t mask_cap_words, void *stream);

/* The steppable engine behind gf2e_scan, for callers that interleave work
 * (the serving loop): one scanner per r keeps `slots` s values resident on
 * the device; submitted s wait in a queue and enter freed slots; each step
 * advances every resident s by one degree (batched launches) and runs the
 * interval-end gcds; finished s are returned by poll with their tags
 * (tag0 + i for the i-th submitted s).  No counterpart in the reference,
 * which scans one s at a time (trinomial_scan.cu:648-689). */
typedef struct gf2e_scanner gf2e_scanner;
int gf2e_scanner_footprint(uint64_t r, int slots, size_t *device_bytes);
int gf2e_scanner_create(uint64_t r, int slots, gf2e_scanner **scanner);
/* Blocked-DDF scanner (see gf2e_scan_blocked); step(degrees) advances
 * ceil(degrees / block) blocks.  block = 1 is gf2e_scanner_create. */
int gf2e_scanner_footprint_blocked(uint64_t r, int slots, int block, size_t *device_bytes);
int gf2e_scanner_create_blocked(uint64_t r, int slots, int block, gf2e_scanner **scanner);
int gf2e_scanner_destroy(gf2e_scanner *scanner);
/* Interval schedule for the jobs submitted after this call (default
 * GF2E_SCHED_DOUBLING). */
int gf2e_scanner_set_schedule(gf2e_scanner *scanner, const gf2e_sched *sched);
int gf2e_scanner_submit(gf2e_scanner *scanner, const uint64_t *s_host, int ns, uint64_t k0,
                        uint64_t maxd, uint64_t L0, uint64_t Lmax, uint64_t tag0);
int gf2e_scanner_step(gf2e_scanner *scanner, int degrees, void *stream);
int gf2e_scanner_status(const gf2e_scanner *scanner, int *queued, int *resident,
                        int *finished, uint64_t *sd_pairs);
int gf2e_scanner_poll(gf2e_scanner *scanner, gf2e_scan_result *results_host,
                      uint64_t *tags_host, uint64_t *masks_host, size_t mask_cap_words,
                      int cap, int *nout);
/* Verified frontier of every resident s: every degree <= k_host[i] is known
 * clear (the last interval gcd that came back 1 ended there; k0 before
 * the first).  A job resubmitted with k0 = that frontier continues the
 * scan, which is what trinomial_scan's resume state records
 * (trinomial_scan.cu:144-170, 262-275). */
int gf2e_scanner_frontiers(const gf2e_scanner *scanner, uint64_t *s_host, uint64_t *k_host,
                           uint64_t *tags_host, int cap, int *nout);
/* Interval gcds the scanner has run and the host wall time spent in them
 * (the gcd calls return when their results are known). */
int gf2e_scanner_gcd_time(const gf2e_scanner *scanner, uint64_t *gcds, double *seconds);

/* ======================================================================
 * (f) Serving: continuous batching of (r, s-set, d-range) search jobs.  No
 * counterpart in the reference.  A job is admitted when its device memory
 * (a scanner for its r, shared by all jobs with that r) fits the budget;
 * admission sieves degrees 2..min(dmax, 24) and queues the survivors on the
 * scanner; step() advances every resident scanner; poll() returns finished
 * jobs and their latency since submit; job_lines() gives one result line per
 * s ("s d p<hex>", "s u" for no factor of degree <= dmax, "s rA-B").
 * ====================================================================== */
typedef struct gf2e_server gf2e_server;
int gf2e_server_create(size_t budget_bytes, int slots_per_r, gf2e_server **server);
/* Server whose scanners run the blocked DDF with `block` degrees per step. */
int gf2e_server_create_blocked(size_t budget_bytes, int slots_per_r, int block,
                               gf2e_server **server);
int gf2e_server_destroy(gf2e_server *server);
int gf2e_server_submit(gf2e_server *server, uint64_t job_id, uint64_t r, const uint64_t *s_host,
                       int ns, uint64_t dmax, uint64_t L0, uint64_t Lmax);
int gf2e_server_step(gf2e_server *server, int degrees, void *stream);
int gf2e_server_status(const gf2e_server *server, int *waiting, int *active, int *finished,
                       size_t *used_bytes);
/* (s, d) pairs the server has worked through so far: sieved (each admitted
 * s times the degrees 2..min(dmax, 24) its sieve covered) and scanned (each
 * resident s times the degrees its deep scan actually stepped, so an s that
 * retired early counts only the degrees it ran). */
int gf2e_server_pairs(const gf2e_server *server, uint64_t *sieved, uint64_t *scanned);
int gf2e_server_poll(gf2e_server *server, uint64_t *job_ids_host, double *latency_s_host,
                     int cap, int *nout);
int gf2e_server_job_lines(gf2e_server *server, uint64_t job_id, char *buf, size_t cap,
                          size_t *needed);
int gf2e_server_release(gf2e_server *server, uint64_t job_id);

/* Host-side resolution of a hit (trinomial_scan.cu:208-235,
 * gf2_gcd_ntl.cpp:68-92): for g whose irreducible factors all have degree in
 * [kmin, kmax], the least such degree and the numerically least factor of it
 * (equal-degree splitting when several share the degree). */
int gf2e_resolve_factor(const uint64_t *g_host, size_t gw, uint64_t kmin, uint64_t kmax,
                        uint64_t *d_out, uint64_t *mask_host, size_t mask_cap_words,
                        size_t *mask_words);

/* ======================================================================
 * TrinGPU context (gf2_trinomial_cuda.h:87-178): F (dA), ACC (dACC),
 * product scratch and an FFT plan for r-bit x r-bit products.
 * ====================================================================== */
typedef struct gf2e_trin gf2e_trin;

int gf2e_trin_create(uint64_t r, gf2e_trin **ctx);        /* TrinGPU::init */
int gf2e_trin_destroy(gf2e_trin *ctx);                    /* TrinGPU::fini */
int gf2e_trin_set_s(gf2e_trin *ctx, uint64_t s);          /* TrinGPU::set_s */
/* Device pointers of F (dA) and ACC (dACC), nw words each; product scratch
 * dT0 (2*nw words); FFT size exponent m of the context's r-bit products
 * (one less than the plain size when they take the wrapped form, as at
 * r = 136279841). */
int gf2e_trin_buffers(gf2e_trin *ctx, uint64_t **dA, uint64_t **dACC,
                      uint64_t **dT0, size_t *nw, int *m);
/* The context's other scratch with the reference's sizes (TrinGPU::dT1,
 * 2*nw words; dFA and dFB, 2^m_full points each) and m_full, the plain FFT
 * size exponent of an r-bit x r-bit product (TrinGPU::m,
 * gf2_trinomial_cuda.h:97-115).  The context's own products overwrite them. */
int gf2e_trin_scratch(gf2e_trin *ctx, uint64_t **dT1, uint64_t **dFA,
                      uint64_t **dFB, int *m_full);
int gf2e_trin_reset_A(gf2e_trin *ctx, void *stream);      /* k_set_x on dA */
int gf2e_trin_reset_acc(gf2e_trin *ctx, void *stream);    /* ACC <- 1 */
int gf2e_trin_square_A(gf2e_trin *ctx, void *stream);     /* dA <- dA^2 mod T */
/* dA <- dA^(2^k) mod T, two squarings per pass over dA (no counterpart in
 * the reference's TrinGPU, whose callers loop over square_A). */
int gf2e_trin_square_A_k(gf2e_trin *ctx, uint64_t k, void *stream);
/* dT0 (2r-1 bits) <- x * y, both r-bit device operands (TrinGPU::mul_dev). */
int gf2e_trin_mul_dev(gf2e_trin *ctx, const uint64_t *x_dev,
                      const uint64_t *y_dev, void *stream);
/* dst <- dT0 mod T where dT0 holds L bits (TrinGPU::reduce). */
int gf2e_trin_reduce_T0(gf2e_trin *ctx, uint64_t *dst_dev, uint64_t L,
                        void *stream);
/* ACC <- ACC * (F + x) mod T (TrinGPU::accumulate). */
int gf2e_trin_accumulate(gf2e_trin *ctx, void *stream);

/* ======================================================================
 * Subquadratic gcd for r-bit operands (half-gcd).  Replaces the interval
 * gcd the reference delegates to NTL at r = 136279841 (GF2X GCD,
 * gf2_gcd_ntl.cpp:32-42; hybrid HGCD gf2_gcd_ntl.cpp:360-452) with the same
 * contract as gf2e_gcd_batch: deg_host[i] = deg gcd (0 means gcd = 1), and
 * the gcd itself in g_dev when it fits g_cap_words.  Operands are read, not
 * modified.  max_parallel <= 1: one job after another.  max_parallel >= 2:
 * lockstep batches of up to max_parallel jobs (at most 64, and as many as
 * device memory holds): one host thread steps every member of a batch
 * through the half-gcd recursion together, each launch (base cases, shifts,
 * products, degree reads, division steps) serving all members with their
 * own sizes, so launches and host round trips per gcd fall by the batch
 * size.  Device memory comes from a private stream-ordered pool (about 40
 * words per operand word per member, plus the transforms of the largest
 * matrix product).  Synchronous: returns when every job is done.  stats (may
 * be NULL) sums the work counters (in a batch, its steps count once).
 * ====================================================================== */
typedef struct gf2e_hgcd_stats {
    int64_t nodes;            /* half-gcd calls */
    int64_t base_cases;       /* one-CTA Lehmer base cases */
    int64_t base_rounds;      /* Lehmer rounds inside them */
    int64_t fft_products;     /* sum-of-two-products done with the FFT */
    int64_t school_products;  /* ... done with the schoolbook kernel */
    int64_t division_steps;
    int64_t probes;           /* device-to-host degree reads */
    int64_t us_base;          /* host wall time (us) in base cases */
    int64_t us_products;      /* ... in matrix products (incl. degree reads) */
    int64_t us_division;      /* ... in division steps */
    int64_t us_small_gcd;     /* ... in the final quadratic gcd */
    int64_t base_cycles_serial;  /* SM cycles of base cases in the serial window phase */
    int64_t base_cycles_total;   /* SM cycles of base cases in total */
} gf2e_hgcd_stats;

int gf2e_gcd_large(const gf2e_gcd_job *jobs, int njobs, int64_t *deg_host,
                   int max_parallel, gf2e_hgcd_stats *stats, void *stream);

/* ======================================================================
 * Tuning and the autotuner.  Replaces the reference's runtime FFT knobs
 * (gf2c_taylor_lv / gf2c_bfly_lv, gf2_cantor_cuda.h:24-60, environment
 * GF2C_TAYLOR_LV / GF2C_BFLY_LV) and tsfactor's "--bench" FFT autotune
 * (tsfactor.cu:1986-2080): every candidate is verified on the device
 * against the default configuration (forward transform word-equal, inverse
 * round trip) before it is timed, the fastest is left active, and its
 * settings are returned (and printed by the Python tool as export lines).
 *
 * The tuning is process-wide.  FFT plans and the sieve read it when they
 * are created / launched, so a change affects plans made afterwards (the
 * internal plan cache is keyed by it).  Environment overrides read on first
 * use: GF2E_FFT_TILE_LOG, GF2E_FFT_CMIN, GF2E_FFT_TAYLOR_LV,
 * GF2E_FFT_BFLY_LV, GF2E_SIEVE_STRIP_LOG.
 * ====================================================================== */
typedef struct gf2e_tune {
    int fft_tile_log;    /* log2 elements per shared-memory tile, 11..13; 0 = by size */
    int fft_cmin;        /* least contiguous columns per tile row: 1, 2, 4, 8, 16; 0 = by size */
    int fft_taylor_lv;   /* Taylor levels fused per register stage, 1..3 */
    int fft_bfly_lv;     /* butterfly levels fused per register stage, 1..3 */
    int sieve_strip_log; /* log2 best[] entries per strip CTA, 10..14 */
} gf2e_tune;

int gf2e_tune_default(gf2e_tune *t);          /* built-in defaults */
int gf2e_tune_get(gf2e_tune *t);              /* current (env applied) */
int gf2e_tune_set(const gf2e_tune *t);        /* validated; INVALID if out of range */

/* FFT autotune at size 2^m: candidates over tile size, column floor and
 * stage depths.  best_ms = fwd + inv time of the winner.  report (may be
 * NULL) receives one line per candidate: "tile cmin tlv blv ms ok". */
int gf2e_fft_autotune(int m, int reps, gf2e_tune *best, double *best_ms,
                      char *report, size_t report_cap);

/* Sieve strip-width autotune: runs gf2e_sieve_run(r, 2, dmax, smax) with
 * each strip width, checks the best[] array is identical to the default's,
 * keeps the fastest.  Needs free device memory for two best[] arrays. */
int gf2e_sieve_autotune(uint64_t r, int dmax, uint64_t smax, int reps,
                        gf2e_tune *best, double *best_ms, char *report,
                        size_t report_cap);

/* gcd interval schedule for the deep scan (trinomial_scan.cu:175 uses
 * L0 = 64 doubling to 4096).  Given the measured cost of one scanned degree
 * (t_degree) and of one interval-end gcd (t_gcd), in any common unit, picks
 * L0 and Lmax (powers of two, L0 <= Lmax) minimising the expected cost of
 * scanning one survivor of a k0-deep sieve up to maxd, under the model that
 * the least factor degree d exceeds D with probability k0 / D.  Pure host
 * arithmetic. */
/* Block size of the blocked DDF (gf2e_scan_blocked): per scanned degree the
 * cost is m squarings (t_sq each, per s) plus one modmul (t_mul) per m
 * degrees, least at m = sqrt(t_mul / t_sq); rounded to even, 2..62. */
int gf2e_scan_choose_block(double t_mul, double t_sq, int *block);

int gf2e_scan_choose_interval(uint64_t k0, uint64_t maxd, double t_degree,
                              double t_gcd, uint64_t *L0, uint64_t *Lmax,
                              double *expected_cost);

#ifdef __cplusplus
}
#endif
#endif /* GF2E_H */
