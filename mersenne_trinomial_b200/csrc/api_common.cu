// api_common.cu -- status strings, error detail, launch-geometry helpers.
#include "gf2e_internal.cuh"

#include <string.h>

namespace gf2e {

static thread_local char g_err[1024];

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!cached[dev]) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
            n = 148;
        cached[dev] = n;
    }
    return cached[dev];
}

int grid_for(size_t work, int threads, int ctas_per_sm) {
    size_t want = (work + (size_t)threads - 1) / (size_t)threads;
    size_t cap = (size_t)sm_count() * (size_t)ctas_per_sm;
    if (want > cap) want = cap;
    if (want < 1) want = 1;
    return (int)want;
}

}  // namespace gf2e

extern "C" {

int gf2e_abi_version(void) { return GF2E_ABI_VERSION; }

const char *gf2e_status_string(int status) {
    switch (status) {
    case GF2E_OK: return "ok";
    case GF2E_ERR_INVALID: return "invalid argument";
    case GF2E_ERR_CUDA: return "CUDA error";
    case GF2E_ERR_NOMEM: return "out of memory / workspace too small";
    case GF2E_ERR_UNSUPPORTED_R: return "gcd(r, 2^d-1) != 1; unsupported r";
    case GF2E_ERR_TIMEOUT: return "device wait timed out";
    case GF2E_ERR_OVERFLOW: return "device queue overflow";
    case GF2E_ERR_INTERNAL: return "internal consistency failure";
    default: return "unknown status";
    }
}

const char *gf2e_last_error(void) { return gf2e::g_err; }

int gf2e_stream_sync(void *stream) {
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    return gf2e::cuda_status(e, "stream sync");
}

}  // extern "C"

extern "C" {

int gf2e_device_alloc(void **ptr, size_t bytes) {
    if (!ptr) return gf2e::invalid("null pointer");
    cudaError_t e = cudaMalloc(ptr, bytes ? bytes : 1);
    if (e == cudaErrorMemoryAllocation) {
        gf2e::set_error("cudaMalloc(%zu): out of memory", bytes);
        cudaGetLastError();
        return GF2E_ERR_NOMEM;
    }
    return gf2e::cuda_status(e, "cudaMalloc");
}

int gf2e_device_free(void *ptr) { return gf2e::cuda_status(cudaFree(ptr), "cudaFree"); }

int gf2e_copy_to_host(void *dst_host, const void *src_dev, size_t bytes, void *stream) {
    cudaError_t e = cudaMemcpyAsync(dst_host, src_dev, bytes, cudaMemcpyDeviceToHost,
                                    (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    return gf2e::cuda_status(e, "copy to host");
}

int gf2e_copy_to_device(void *dst_dev, const void *src_host, size_t bytes, void *stream) {
    cudaError_t e = cudaMemcpyAsync(dst_dev, src_host, bytes, cudaMemcpyHostToDevice,
                                    (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    return gf2e::cuda_status(e, "copy to device");
}

}  // extern "C"
