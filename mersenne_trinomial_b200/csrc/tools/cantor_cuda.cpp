// cantor_cuda -- drop-in for the reference tool of the same name
// (cantor_cuda.cu main, 103-189) on libgf2e.so.
//
//   cantor_cuda selftest         transform round trips and linearity, products
//                                 checked by residues mod degree-61 irreducibles
//                                 and against a product at a larger FFT size
//   cantor_cuda bench [bits]     one bits x bits multiply (default 136279841),
//                                 timed, verified by residues (cantor_cuda.cu:160-186)
#include <cinttypes>
#include <chrono>
#include <cstring>
#include <vector>

#include "gf2e_cantor.hpp"

static double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

static u64 rng_state = 0x9E3779B97F4A7C15ULL;
static u64 rnd() {
    u64 z = (rng_state += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
static void rand_bits(std::vector<u64> &v, u64 bits) {
    v.assign(bits_to_words(bits), 0);
    for (auto &w : v) w = rnd();
    if (bits & 63) v.back() &= (~0ULL) >> (64 - (bits & 63));
}

// residues mod an irreducible q of degree 61 (gf2_cantor_engine.h:278-325)
struct Res61 {
    u64 q;
    static const int d = 61;
    u64 mul(u64 a, u64 b) const {
        u64 lo = 0, hi = 0;
        for (int i = 0; i < 64; i++)
            if ((b >> i) & 1) { lo ^= a << i; if (i) hi ^= a >> (64 - i); }
        for (int bit = 2 * d - 2; bit >= d; bit--) {
            u64 have = ((bit >= 64 ? hi : lo) >> (bit & 63)) & 1;
            if (!have) continue;
            int sh = bit - d;
            lo ^= q << sh;
            if (sh) hi ^= q >> (64 - sh);
        }
        return lo;
    }
    u64 red(u64 v) const {
        for (int bit = 63; bit >= d; bit--)
            if ((v >> bit) & 1) v ^= q << (bit - d);
        return v;
    }
    u64 residue(const u64 *a, u64 bits) const {
        u64 x64 = 1, base = 2;
        for (int e = 64; e; e >>= 1) {           // x^64
            if (e & 1) x64 = mul(x64, base);
            base = mul(base, base);
        }
        u64 r = 0;
        for (size_t w = bits_to_words(bits); w-- > 0;) r = mul(r, x64) ^ red(a[w]);
        return r;
    }
    static Res61 find(u64 seed) {
        Res61 p;
        for (u64 low = seed | 1;; low += 2) {
            p.q = (1ULL << 61) | (low & ((1ULL << 61) - 1));
            u64 t = 2;
            for (int i = 0; i < 61; i++) t = p.mul(t, t);
            if (t == 2) return p;
        }
    }
};

static bool check_residues(const std::vector<u64> &a, u64 ab, const std::vector<u64> &b, u64 bb,
                           const std::vector<u64> &c) {
    bool ok = true;
    const u64 seeds[3] = {0x1234567ULL, 0xDEADBEEFULL, 0xC0FFEEULL};
    for (u64 sd : seeds) {
        Res61 p = Res61::find(sd);
        ok &= p.mul(p.residue(a.data(), ab), p.residue(b.data(), bb)) ==
              p.residue(c.data(), ab + bb);
    }
    return ok;
}

int main(int argc, char **argv) {
    const char *mode = argc > 1 ? argv[1] : "selftest";
    CantorBasis B;
    B.build();
    if (!strcmp(mode, "selftest")) {
        int bad = 0;
        for (int m = 1; m <= 22; m += (m < 12 ? 1 : 5)) {
            size_t n = (size_t)1 << m;
            std::vector<u64> f(n), g(n), h(n), out(n);
            for (size_t i = 0; i < n; i++) { f[i] = rnd(); g[i] = rnd(); h[i] = f[i] ^ g[i]; }
            CudaFFT F;
            F.init(m, B);
            void *df, *dg, *dh;
            gf2e_or_die(gf2e_device_alloc(&df, n * 8), "alloc");
            gf2e_or_die(gf2e_device_alloc(&dg, n * 8), "alloc");
            gf2e_or_die(gf2e_device_alloc(&dh, n * 8), "alloc");
            gf2e_copy_to_device(df, f.data(), n * 8, nullptr);
            gf2e_copy_to_device(dg, g.data(), n * 8, nullptr);
            gf2e_copy_to_device(dh, h.data(), n * 8, nullptr);
            F.fwd((u64 *)df); F.fwd((u64 *)dg); F.fwd((u64 *)dh);
            std::vector<u64> tf(n), tg(n), th(n);
            gf2e_copy_to_host(tf.data(), df, n * 8, nullptr);
            gf2e_copy_to_host(tg.data(), dg, n * 8, nullptr);
            gf2e_copy_to_host(th.data(), dh, n * 8, nullptr);
            bool lin = true;
            for (size_t i = 0; i < n; i++) lin &= (tf[i] ^ tg[i]) == th[i];
            F.inv((u64 *)df);
            gf2e_copy_to_host(out.data(), df, n * 8, nullptr);
            bool rt = out == f;
            printf("m=%2d  linearity %s  roundtrip %s\n", m, lin ? "PASS" : "FAIL",
                   rt ? "PASS" : "FAIL");
            bad += !lin || !rt;
            gf2e_device_free(df); gf2e_device_free(dg); gf2e_device_free(dh);
            F.fini();
        }
        u64 sizes[][2] = {{1, 1}, {100, 77}, {4096, 4096}, {100000, 100000},
                          {1048576, 524288}, {8000000, 8000000}};
        for (auto &sz : sizes) {
            std::vector<u64> a, b;
            rand_bits(a, sz[0]);
            rand_bits(b, sz[1]);
            std::vector<u64> c(mul_out_words(sz[0], sz[1]));
            gf2x_fft_mul(a.data(), sz[0], b.data(), sz[1], c.data(), B);
            bool ok = check_residues(a, sz[0], b, sz[1], c);
            printf("mul %8" PRIu64 " x %8" PRIu64 " bits: %s\n", sz[0], sz[1], ok ? "PASS" : "FAIL");
            bad += !ok;
        }
        printf(bad ? "\nGPU SELFTEST: %d FAILURES\n" : "\nGPU SELFTEST: ALL PASS\n", bad);
        return bad ? 1 : 0;
    }
    if (!strcmp(mode, "bench")) {
        u64 nb = 136279841ULL;
        for (int i = 2; i < argc; i++)
            if (strcmp(argv[i], "legacy") && strcmp(argv[i], "--legacy")) nb = strtoull(argv[i], 0, 10);
        std::vector<u64> a, b;
        rand_bits(a, nb);
        rand_bits(b, nb);
        std::vector<u64> out(mul_out_words(nb, nb));
        double t0 = now_s();
        gf2x_fft_mul(a.data(), nb, b.data(), nb, out.data(), B);
        printf("GPU multiply (%" PRIu64 " x %" PRIu64 " bits, FFT 2^%d) incl. transfers: %.1f ms\n",
               nb, nb, gf2e_mul_fft_m(nb, nb), (now_s() - t0) * 1e3);
        bool ok = check_residues(a, nb, b, nb, out);
        printf("residue checks: %s\n", ok ? "PASS" : "FAIL");
        return ok ? 0 : 1;
    }
    fprintf(stderr, "usage: %s selftest | bench [bits]\n", argv[0]);
    return 1;
}
