// gf2e_trinomial.hpp -- drop-in for the reference's gf2_trinomial_cuda.h
// TrinGPU context (gf2_trinomial_cuda.h:87-178), routed to libgf2e.so.
// Member names and meaning follow the reference: dA holds F_k = x^(2^k) mod
// T, dACC the running product, dT0 a 2r-bit product; nw words per residue.
#pragma once
#include <algorithm>

#include "gf2e_cantor.hpp"

// gf2_trinomial_cuda.h:22-30
static inline u64 spread32(u32 v) {
    u64 x = v;
    x = (x | (x << 16)) & 0x0000FFFF0000FFFFULL;
    x = (x | (x << 8)) & 0x00FF00FF00FF00FFULL;
    x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0FULL;
    x = (x | (x << 2)) & 0x3333333333333333ULL;
    x = (x | (x << 1)) & 0x5555555555555555ULL;
    return x;
}

// Members as in the reference: Bb the Cantor basis, F a transform plan of
// 2^m points (m the plain FFT size of an r-bit x r-bit product), dT1 a
// second 2r-bit scratch, dFA and dFB transform buffers of F.n points.  The
// context's own products (mul_dev, accumulate) use dT0, dT1, dFA and dFB
// as scratch, as the reference's do.
struct TrinGPU {
    u64 r = 0, s = 0;
    size_t nw = 0, nw2 = 0;
    int m = 0;
    CantorBasis Bb;
    CudaFFT F;
    u64 *dA = nullptr, *dACC = nullptr, *dT0 = nullptr, *dT1 = nullptr;
    u64 *dFA = nullptr, *dFB = nullptr;
    gf2e_trin *ctx = nullptr;

    void init(u64 r_) {
        r = r_;
        s = 0;
        gf2e_or_die(gf2e_trin_create(r, &ctx), "TrinGPU::init");
        int m_ctx = 0;
        gf2e_or_die(gf2e_trin_buffers(ctx, &dA, &dACC, &dT0, &nw, &m_ctx), "TrinGPU::init");
        gf2e_or_die(gf2e_trin_scratch(ctx, &dT1, &dFA, &dFB, &m), "TrinGPU::init");
        nw2 = 2 * nw;
        Bb.build();
        F.init(m, Bb);
    }
    void set_s(u64 s_) {
        if (!(s_ >= 1 && 2 * s_ < r)) {
            fprintf(stderr, "need 1 <= s <= (r-1)/2\n");
            exit(1);
        }
        gf2e_or_die(gf2e_trin_set_s(ctx, s_), "TrinGPU::set_s");
        s = s_;
    }
    void set_x() { gf2e_or_die(gf2e_trin_reset_A(ctx, nullptr), "k_set_x"); }
    void reset_acc() { gf2e_or_die(gf2e_trin_reset_acc(ctx, nullptr), "TrinGPU::reset_acc"); }
    void fini() {
        if (ctx) gf2e_trin_destroy(ctx);
        ctx = nullptr;
        F.fini();
        dA = dACC = dT0 = dT1 = dFA = dFB = nullptr;
    }
    void reduce(u64 *dst_rbits, u64 L) {
        gf2e_or_die(gf2e_trin_reduce_T0(ctx, dst_rbits, L, nullptr), "TrinGPU::reduce");
    }
    void square_A() { gf2e_or_die(gf2e_trin_square_A(ctx, nullptr), "TrinGPU::square_A"); }
    // k squarings of dA, two per pass (an addition to the reference's TrinGPU)
    void square_A_k(u64 k) {
        gf2e_or_die(gf2e_trin_square_A_k(ctx, k, nullptr), "TrinGPU::square_A_k");
    }
    void mul_dev(const u64 *dx, const u64 *dy) {
        gf2e_or_die(gf2e_trin_mul_dev(ctx, dx, dy, nullptr), "TrinGPU::mul_dev");
    }
    void accumulate() { gf2e_or_die(gf2e_trin_accumulate(ctx, nullptr), "TrinGPU::accumulate"); }
};

// gf2_trinomial_cuda.h:182-198: the reference's CPU checks, v mod T for a
// polynomial of `bits` bits (bits <= 2r - 1) and a <- a^2 mod T, computed
// here on the GPU (fold reduction, single-pass squaring).  v and a hold
// at least ceil(r/64) words; v keeps its length, its words above r zeroed.
static inline void cpu_mod_trinomial(std::vector<u64> &v, u64 bits, u64 r, u64 s) {
    if (bits <= r) return;
    if (bits > 2 * r - 1) {
        fprintf(stderr, "cpu_mod_trinomial: %llu bits > 2r-1\n", (unsigned long long)bits);
        exit(1);
    }
    const size_t pw = bits_to_words(bits), nw = bits_to_words(r);
    gf2e_dev_words dp, dr;
    dp.ensure(pw);
    dr.ensure(nw);
    gf2e_or_die(gf2e_copy_to_device(dp.get(), v.data(), pw * 8, nullptr), "upload");
    gf2e_or_die(gf2e_trin_reduce(dp.get(), bits, dr.get(), r, s, nullptr), "cpu_mod_trinomial");
    std::vector<u64> red(nw);
    gf2e_or_die(gf2e_copy_to_host(red.data(), dr.get(), nw * 8, nullptr), "download");
    std::fill(v.begin(), v.end(), 0);
    std::copy(red.begin(), red.end(), v.begin());
}
static inline void cpu_square_mod(std::vector<u64> &a, u64 r, u64 s) {
    const size_t nw = bits_to_words(r);
    a.resize(nw);
    gf2e_dev_words din, dout;
    din.ensure(nw);
    dout.ensure(nw);
    gf2e_or_die(gf2e_copy_to_device(din.get(), a.data(), nw * 8, nullptr), "upload");
    gf2e_or_die(gf2e_trin_square(din.get(), dout.get(), r, s, nullptr), "cpu_square_mod");
    gf2e_or_die(gf2e_copy_to_host(a.data(), dout.get(), nw * 8, nullptr), "download");
}
