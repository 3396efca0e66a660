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
#include <cstring>
#include <memory>
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

// A device buffer of u64 words owned by a shared handle (freed with the last
// copy of the object holding it).
struct gf2e_dev_words {
    std::shared_ptr<void> p;
    size_t words = 0;
    u64 *get() const { return (u64 *)p.get(); }
    void ensure(size_t w) {
        if (words >= w) return;
        void *d = nullptr;
        gf2e_or_die(gf2e_device_alloc(&d, (w ? w : 1) * 8), "device allocation");
        p = std::shared_ptr<void>(d, [](void *q) { gf2e_device_free(q); });
        words = w;
    }
};

// gf2_cantor_cuda.h:361-521 (device buffers of n u64, in place).  dW holds
// the n/2 twiddles W[t] on the device, as the reference's CudaFFT::dW
// (gf2_cantor_cuda.h:364-377); the library's transforms rebuild them from
// byte tables and do not read dW.
struct CudaFFT {
    int m = 0;
    size_t n = 0;
    gf2e_fft_plan *plan = nullptr;
    u64 *dW = nullptr;
    void init(int m_, const CantorBasis &) {
        m = m_;
        n = (size_t)1 << m;
        gf2e_or_die(gf2e_fft_plan_create(m, &plan), "CudaFFT::init");
        std::vector<u64> W = twiddles();
        void *d = nullptr;
        gf2e_or_die(gf2e_device_alloc(&d, W.size() * 8), "CudaFFT::init dW");
        gf2e_or_die(gf2e_copy_to_device(d, W.data(), W.size() * 8, nullptr), "CudaFFT::init dW");
        dW = (u64 *)d;
    }
    void fini() {
        if (plan) gf2e_fft_plan_destroy(plan);
        if (dW) gf2e_device_free(dW);
        plan = nullptr;
        dW = nullptr;
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

// gf2_cantor_engine.h:125-187: the transform on host buffers of n = 2^m
// points (natural order in and out), computed on the GPU: fwd / inv move
// the buffer to the device, transform it there and copy it back.  W holds
// the reference's twiddles W[t], t < n/2.  Copies share the plan.
struct CantorFFT {
    int m = 0;
    size_t n = 0;
    std::vector<u64> W;
    std::shared_ptr<gf2e_fft_plan> plan;
    mutable gf2e_dev_words buf;

    void init(int m_, const CantorBasis &) {
        m = m_;
        n = (size_t)1 << m;
        gf2e_fft_plan *p = nullptr;
        gf2e_or_die(gf2e_fft_plan_create(m, &p), "CantorFFT::init");
        plan = std::shared_ptr<gf2e_fft_plan>(p, [](gf2e_fft_plan *q) { gf2e_fft_plan_destroy(q); });
        W.assign(n > 1 ? n / 2 : 1, 0);
        gf2e_or_die(gf2e_fft_twiddles(p, W.data()), "CantorFFT::init twiddles");
        W.resize(n >> 1);
    }
    void fwd(u64 *f) const { run(f, true); }
    void inv(u64 *f) const { run(f, false); }

  private:
    void run(u64 *f, bool forward) const {
        buf.ensure(n);
        gf2e_or_die(gf2e_copy_to_device(buf.get(), f, n * 8, nullptr), "CantorFFT upload");
        gf2e_or_die(forward ? gf2e_fft_fwd(plan.get(), buf.get(), nullptr)
                            : gf2e_fft_inv(plan.get(), buf.get(), nullptr),
                    forward ? "CantorFFT::fwd" : "CantorFFT::inv");
        gf2e_or_die(gf2e_copy_to_host(f, buf.get(), n * 8, nullptr), "CantorFFT download");
    }
};

// gf2_cantor_engine.h:207-229: host operands, host scratch FA and FB of F.n
// words each.  The product runs on the GPU; on return out holds the
// mul_out_words(abits, bbits) product words, FA the inverse transform (the
// product's 32-bit chunk coefficients) and FB the transform of b, as in the
// reference.  A transform too small for the product prints "FFT too small"
// and exits(1), as the reference does.
static inline void gf2x_fft_mul_buf(const u64 *a, u64 abits, const u64 *b, u64 bbits, u64 *out,
                                    const CantorFFT &F, u64 *FA, u64 *FB) {
    const size_t ca = (size_t)((abits + 31) >> 5), cb = (size_t)((bbits + 31) >> 5);
    if (ca + cb - 1 > F.n) {
        fprintf(stderr, "FFT too small\n");
        exit(1);
    }
    const size_t wa = bits_to_words(abits), wb = bits_to_words(bbits);
    const size_t ow = mul_out_words(abits, bbits);
    gf2e_dev_words da, db, dout, fa, fb;
    da.ensure(wa); db.ensure(wb); dout.ensure(ow); fa.ensure(F.n); fb.ensure(F.n);
    gf2e_or_die(gf2e_copy_to_device(da.get(), a, wa * 8, nullptr), "upload");
    gf2e_or_die(gf2e_copy_to_device(db.get(), b, wb * 8, nullptr), "upload");
    gf2e_or_die(gf2e_mul(F.plan.get(), da.get(), abits, db.get(), bbits, dout.get(), fa.get(),
                         fb.get(), nullptr), "gf2x_fft_mul_buf");
    gf2e_or_die(gf2e_copy_to_host(out, dout.get(), ow * 8, nullptr), "download");
    gf2e_or_die(gf2e_copy_to_host(FA, fa.get(), F.n * 8, nullptr), "download");
    gf2e_or_die(gf2e_copy_to_host(FB, fb.get(), F.n * 8, nullptr), "download");
}

// gf2_cantor_cuda.h:114-156: the element-wise kernels of a product, as
// host calls on device buffers (a reference translation unit drops the
// launch configuration: k_pack<<<b, t>>>(...) becomes k_pack(...)).
static inline void k_pack(const u64 *a, size_t nwords, u64 *F, size_t nchunks, size_t n) {
    gf2e_or_die(gf2e_fft_pack(a, nwords, F, nchunks, n, nullptr), "k_pack");
}
static inline void k_pointwise(u64 *fa, const u64 *fb, size_t n) {
    gf2e_or_die(gf2e_fft_pointwise(fa, fb, n, nullptr), "k_pointwise");
}
static inline void k_overlap_add(const u64 *F, size_t nchunks, u64 *out, size_t owords) {
    gf2e_or_die(gf2e_fft_overlap_add(F, nchunks, out, owords, nullptr), "k_overlap_add");
}

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

// gf2_cantor_engine.h:247-274: the reference's schoolbook products (its
// oracles for the transform).  Here they are the same product, computed on
// the GPU like gf2x_fft_mul: out gets mul_out_words(abits, bbits) words.
static inline void gf2x_naive_mul(const u64 *a, u64 abits, const u64 *b, u64 bbits, u64 *out) {
    gf2x_fft_mul(a, abits, b, bbits, out, CantorBasis());
}
static inline void gf2x_comb_mul(const u64 *a, u64 abits, const u64 *b, u64 bbits, u64 *out) {
    gf2x_fft_mul(a, abits, b, bbits, out, CantorBasis());
}

// gf2_cantor_engine.h:278-334: residues modulo an irreducible q of degree
// d <= 62 over GF(2), the reference's check of big products (a product's
// residue equals the product of the operands' residues).  Host arithmetic:
// shift-and-add products reduced one bit at a time.
struct ModP {
    u64 q = 0;
    int d = 0;
    u64 mulx(u64 a) const {                       // a * x mod q
        a <<= 1;
        return ((a >> d) & 1) ? a ^ q : a;
    }
    u64 mul(u64 a, u64 b) const {                 // a * b mod q, a, b < 2^d
        u64 r = 0;
        for (; b; b >>= 1) {
            if (b & 1) r ^= a;
            a = mulx(a);
        }
        return r;
    }
    u64 red64(u64 v) const {                      // v mod q for any 64-bit v
        for (int bit = 63; bit >= d; bit--)
            if ((v >> bit) & 1) v ^= q << (bit - d);
        return v;
    }
    u64 pw(u64 a, u64 e) const {
        u64 r = 1;
        for (; e; e >>= 1) {
            if (e & 1) r = mul(r, a);
            a = mul(a, a);
        }
        return r;
    }
    // Rabin's test: x^(2^d) = x mod q, and gcd(x^(2^(d/p)) - x, q) = 1 for
    // every prime p dividing d.  For prime d (the reference's d = 61) the
    // gcd condition is x^2 != x, so the reference's search (the first q
    // from the seed for which its test holds) finds the same q.
    bool irreducible() const {
        std::vector<u64> frob(d + 1);
        frob[0] = 2;
        for (int i = 1; i <= d; i++) frob[i] = mul(frob[i - 1], frob[i - 1]);
        if (frob[d] != 2) return false;
        int left = d;
        for (int p = 2; p <= left; p++) {
            if (left % p) continue;
            while (left % p == 0) left /= p;
            u64 g = frob[d / p] ^ 2, h = q;       // gcd(x^(2^(d/p)) + x, q)
            while (g) {
                int dg = 63 - __builtin_clzll(g);
                while (h && 63 - __builtin_clzll(h) >= dg)
                    h ^= g << ((63 - __builtin_clzll(h)) - dg);
                u64 t = g; g = h; h = t;
            }
            if (h != 1) return false;
        }
        return true;
    }
    // a (abits bits) mod q: Horner over 64-bit words from the top
    u64 residue(const u64 *a, u64 abits) const {
        const u64 x64 = pw(2, 64);
        u64 r = 0;
        for (size_t w = bits_to_words(abits); w-- > 0;) r = mul(r, x64) ^ red64(a[w]);
        return r;
    }
};

// the first irreducible q = x^d + (low | 1) for low = seed, seed + 2, ...
// (gf2_cantor_engine.h:327-334)
static inline ModP find_irreducible_modp(int d, u64 seed) {
    ModP p;
    p.d = d;
    for (u64 low = seed | 1;; low += 2) {
        p.q = ((u64)1 << d) | (low & (((u64)1 << d) - 1));
        if (p.irreducible()) return p;
    }
}
