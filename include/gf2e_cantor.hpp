// gf2e_cantor.hpp -- drop-in for the reference's gf2_cantor_engine.h /
// gf2_cantor_cuda.h entry points, routed to libgf2e.so (GPU).  A reference
// translation unit replaces
//     #include "gf2_cantor_cuda.h"      (or gf2_cantor_engine.h)
// with
//     #include "gf2e_cantor.hpp"
// and links -lgf2e.  Names and argument meaning are the reference's; a
// non-zero library status prints the detail and exits(1), as the
// reference's CUCHK does (gf2_cantor_cuda.h:65-69).
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "gf2e.h"

typedef uint64_t u64;
typedef uint32_t u32;

inline void gf2e_or_die(int st, const char *what) {
    if (st != GF2E_OK) {
        fprintf(stderr, "%s: %s (%s)\n", what, gf2e_status_string(st), gf2e_last_error());
        exit(1);
    }
}

// gf2_cantor_engine.h:192-203
static inline size_t bits_to_words(u64 bits) { return (size_t)((bits + 63) >> 6); }
static inline size_t mul_out_words(u64 abits, u64 bbits) {
    return gf2e_mul_out_words(abits, bbits);
}
static inline u32 get_chunk(const u64 *a, size_t nwords, size_t k) {
    size_t pos = 32 * k, w = pos >> 6;
    if (w >= nwords) return 0;
    return (u32)(a[w] >> (pos & 63));
}

// gf2_cantor_engine.h:74-121
struct CantorBasis {
    u64 b[64];
    int len = 0;
    void build() { gf2e_or_die(gf2e_cantor_basis(b, &len), "CantorBasis::build"); }
    bool verify() const { return len == 64 && b[0] == 1; }
};

// gf2_cantor_cuda.h:361-521 (device buffers of n u64, in place)
struct CudaFFT {
    int m = 0;
    size_t n = 0;
    gf2e_fft_plan *plan = nullptr;
    void init(int m_, const CantorBasis &) {
        m = m_;
        n = (size_t)1 << m;
        gf2e_or_die(gf2e_fft_plan_create(m, &plan), "CudaFFT::init");
    }
    void fini() {
        if (plan) gf2e_fft_plan_destroy(plan);
        plan = nullptr;
    }
    void fwd(u64 *df) const { gf2e_or_die(gf2e_fft_fwd(plan, df, nullptr), "CudaFFT::fwd"); }
    void inv(u64 *df) const { gf2e_or_die(gf2e_fft_inv(plan, df, nullptr), "CudaFFT::inv"); }
    std::vector<u64> twiddles() const {
        std::vector<u64> W(n > 1 ? n / 2 : 1);
        gf2e_or_die(gf2e_fft_twiddles(plan, W.data()), "CudaFFT::twiddles");
        return W;
    }
    static void launch_dims(size_t work, int &blocks, int &threads) {
        threads = 256;
        size_t b = (work + 255) / 256;
        blocks = (int)(b > 65535 ? 65535 : (b ? b : 1));
    }
};

// gf2_cantor_engine.h:207-229: device operands and scratch
static inline void gf2x_fft_mul_buf_dev(const u64 *a, u64 abits, const u64 *b, u64 bbits,
                                        u64 *out, const CudaFFT &F, u64 *FA, u64 *FB) {
    gf2e_or_die(gf2e_mul(F.plan, a, abits, b, bbits, out, FA, FB, nullptr), "gf2x_fft_mul");
}

// gf2_cantor_engine.h:232-242: host operands, out = mul_out_words words
static inline void gf2x_fft_mul(const u64 *a, u64 abits, const u64 *b, u64 bbits, u64 *out,
                                const CantorBasis &) {
    int m = gf2e_mul_fft_m(abits, bbits);
    gf2e_fft_plan *plan = nullptr;
    gf2e_or_die(gf2e_fft_plan_create(m, &plan), "gf2x_fft_mul plan");
    size_t wa = bits_to_words(abits), wb = bits_to_words(bbits), ow = mul_out_words(abits, bbits);
    size_t n = (size_t)1 << m;
    void *da, *db, *dout, *fa, *fb;
    gf2e_or_die(gf2e_device_alloc(&da, wa * 8), "alloc");
    gf2e_or_die(gf2e_device_alloc(&db, wb * 8), "alloc");
    gf2e_or_die(gf2e_device_alloc(&dout, ow * 8), "alloc");
    gf2e_or_die(gf2e_device_alloc(&fa, n * 8), "alloc");
    gf2e_or_die(gf2e_device_alloc(&fb, n * 8), "alloc");
    gf2e_or_die(gf2e_copy_to_device(da, a, wa * 8, nullptr), "upload");
    gf2e_or_die(gf2e_copy_to_device(db, b, wb * 8, nullptr), "upload");
    gf2e_or_die(gf2e_mul(plan, (u64 *)da, abits, (u64 *)db, bbits, (u64 *)dout, (u64 *)fa,
                         (u64 *)fb, nullptr), "gf2x_fft_mul");
    gf2e_or_die(gf2e_copy_to_host(out, dout, ow * 8, nullptr), "download");
    gf2e_device_free(da); gf2e_device_free(db); gf2e_device_free(dout);
    gf2e_device_free(fa); gf2e_device_free(fb);
    gf2e_fft_plan_destroy(plan);
}
