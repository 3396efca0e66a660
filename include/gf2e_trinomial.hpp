// gf2e_trinomial.hpp -- drop-in for the reference's gf2_trinomial_cuda.h
// TrinGPU context (gf2_trinomial_cuda.h:87-178), routed to libgf2e.so.
// Member names and meaning follow the reference: dA holds F_k = x^(2^k) mod
// T, dACC the running product, dT0 a 2r-bit product; nw words per residue.
#pragma once
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

struct TrinGPU {
    u64 r = 0, s = 0;
    size_t nw = 0, nw2 = 0;
    int m = 0;
    u64 *dA = nullptr, *dACC = nullptr, *dT0 = nullptr;
    gf2e_trin *ctx = nullptr;

    void init(u64 r_) {
        r = r_;
        s = 0;
        gf2e_or_die(gf2e_trin_create(r, &ctx), "TrinGPU::init");
        gf2e_or_die(gf2e_trin_buffers(ctx, &dA, &dACC, &dT0, &nw, &m), "TrinGPU::init");
        nw2 = 2 * nw;
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
    }
    void reduce(u64 *dst_rbits, u64 L) {
        gf2e_or_die(gf2e_trin_reduce_T0(ctx, dst_rbits, L, nullptr), "TrinGPU::reduce");
    }
    void square_A() { gf2e_or_die(gf2e_trin_square_A(ctx, nullptr), "TrinGPU::square_A"); }
    void mul_dev(const u64 *dx, const u64 *dy) {
        gf2e_or_die(gf2e_trin_mul_dev(ctx, dx, dy, nullptr), "TrinGPU::mul_dev");
    }
    void accumulate() { gf2e_or_die(gf2e_trin_accumulate(ctx, nullptr), "TrinGPU::accumulate"); }
};
