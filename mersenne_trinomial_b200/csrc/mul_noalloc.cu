// mul_noalloc.cu -- GF(2)[x] product that allocates no memory per call.
//
// Some callers of this library cannot allocate device memory while they
// run: a serving process that reserves its whole HBM budget when it starts
// and admits work against that budget, or a host loop that must not let an
// allocator call synchronise the device between its launches.  For them,
// gf2e_mul_noalloc keeps the transform scratch (two buffers of up to 2^18
// u64 points) and the twiddle byte tables in fixed arrays of this file.
// Every GPU that loads the library holds these 4 MiB + 8 KiB until the
// process exits.
//
// The fixed arrays are host-side stand-ins in host code; their device
// addresses come from cudaGetSymbolAddress, taken once per device, with that
// device current, by the set-up in the first call on that device (which also
// fills the twiddle tables and builds the pass schedules on the host).  The
// set-up is published with release/acquire ordering, so a thread that sees a
// device as ready also sees its addresses and plans.  A cudaDeviceReset
// reloads the module and drops what the set-up uploaded; calls after one in
// the same process are not supported.
#include "gf2e_internal.cuh"

#include <atomic>
#include <mutex>

namespace gf2e {
int mul(const gf2e_fft_plan *plan, const u64 *a, u64 abits, const u64 *b, u64 bbits,
        u64 *out, u64 *fa, u64 *fb, cudaStream_t st);
int mul_fft_m(u64 abits, u64 bbits);
int fft_plan_create_tables(int m, const u64 *tab_dev, gf2e_fft_plan **out);
void twiddle_byte_tables(u64 *tab);
int twiddle_table_words();
}  // namespace gf2e

namespace {

constexpr int MAX_M = GF2E_MUL_NOALLOC_MAX_M;
constexpr int TAB_WORDS = 4 * 256;

// scratch for the two operand transforms: FA = [0, 2^m), FB = [2^m, 2^(m+1))
static __device__ __align__(256) uint64_t g_noalloc_scratch[2ull << MAX_M];
static __device__ __align__(256) uint64_t g_noalloc_twiddles[TAB_WORDS];

struct DeviceState {
    std::atomic<bool> ready{false};
    u64 *scratch = nullptr;      // device address of g_noalloc_scratch
    u64 *twiddles = nullptr;     // device address of g_noalloc_twiddles
    gf2e_fft_plan *plan[MAX_M + 1] = {};
};

DeviceState g_state[64];
std::mutex g_mu;

int setup_device(int dev) {
    DeviceState &d = g_state[dev];
    cudaError_t e = cudaGetSymbolAddress((void **)&d.scratch, g_noalloc_scratch);
    if (e != cudaSuccess) return gf2e::cuda_status(e, "noalloc scratch address");
    e = cudaGetSymbolAddress((void **)&d.twiddles, g_noalloc_twiddles);
    if (e != cudaSuccess) return gf2e::cuda_status(e, "noalloc twiddle address");
    if (gf2e::twiddle_table_words() != TAB_WORDS)
        return gf2e::invalid("twiddle table size mismatch");
    u64 host_tab[TAB_WORDS];
    gf2e::twiddle_byte_tables(host_tab);
    e = cudaMemcpyToSymbol(g_noalloc_twiddles, host_tab, sizeof host_tab);
    if (e != cudaSuccess) return gf2e::cuda_status(e, "noalloc twiddle upload");
    // plans go into a local table first: a failure part way destroys the
    // ones already made, and the next call starts the set-up afresh
    gf2e_fft_plan *plans[MAX_M + 1] = {};
    for (int m = 1; m <= MAX_M; m++) {
        int st = gf2e::fft_plan_create_tables(m, d.twiddles, &plans[m]);
        if (st != GF2E_OK) {
            for (int k = 1; k < m; k++) gf2e_fft_plan_destroy(plans[k]);
            return st;
        }
    }
    for (int m = 1; m <= MAX_M; m++) d.plan[m] = plans[m];
    d.ready.store(true, std::memory_order_release);
    return GF2E_OK;
}

}  // namespace

extern "C" {

int gf2e_mul_noalloc(const uint64_t *a_dev, uint64_t abits, const uint64_t *b_dev,
                     uint64_t bbits, uint64_t *out_dev, void *stream) {
    if (!a_dev || !b_dev || !out_dev) return gf2e::invalid("gf2e_mul_noalloc: null argument");
    if (abits == 0 || bbits == 0) return gf2e::invalid("gf2e_mul_noalloc: empty operand");
    const int m = gf2e::mul_fft_m(abits, bbits);
    if (m > MAX_M)
        return gf2e::invalid(
            "gf2e_mul_noalloc: %llu x %llu bits needs a transform of 2^%d points; the fixed "
            "scratch holds 2^%d (ceil(abits/32) + ceil(bbits/32) - 1 <= %llu)",
            (unsigned long long)abits, (unsigned long long)bbits, m, MAX_M,
            (unsigned long long)(1ull << MAX_M));
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return gf2e::cuda_status(e, "cudaGetDevice");
    if (dev < 0 || dev >= 64) return gf2e::invalid("device index %d out of range", dev);
    if (!g_state[dev].ready.load(std::memory_order_acquire)) {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_state[dev].ready.load(std::memory_order_acquire)) GF2E_TRY(setup_device(dev));
    }
    const DeviceState &d = g_state[dev];
    // the first forward pass writes every point of FA and FB (operand chunks,
    // zeros above them), so nothing left by an earlier call is read
    u64 *fa = d.scratch, *fb = d.scratch + ((size_t)1 << m);
    return gf2e::mul(d.plan[m], a_dev, abits, b_dev, bbits, out_dev, fa, fb,
                     (cudaStream_t)stream);
}

}  // extern "C"
