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

// residues mod irreducibles of degree 61 (ModP, gf2_cantor_engine.h:278-334):
// a product's residue must be the product of its operands' residues
static const u64 kResidueSeeds[3] = {0x1234567ULL, 0xDEADBEEFULL, 0xC0FFEEULL};

static bool check_residues(const std::vector<u64> &a, u64 ab, const std::vector<u64> &b, u64 bb,
                           const std::vector<u64> &c, bool print) {
    bool ok = true;
    for (u64 sd : kResidueSeeds) {
        ModP p = find_irreducible_modp(61, sd);
        const bool good = p.mul(p.residue(a.data(), ab), p.residue(b.data(), bb)) ==
                          p.residue(c.data(), ab + bb - 1);
        if (print) printf("residue check mod 0x%" PRIx64 ": %s\n", p.q, good ? "PASS" : "FAIL");
        ok &= good;
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
            bool ok = check_residues(a, sz[0], b, sz[1], c, false);
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
        printf("transform path: FUSED\n");
        double t0 = now_s();
        gf2x_fft_mul(a.data(), nb, b.data(), nb, out.data(), B);
        printf("wall including transfers/alloc: %.2fs\n", now_s() - t0);
        return check_residues(a, nb, b, nb, out, true) ? 0 : 1;
    }
    fprintf(stderr, "usage: %s selftest | bench [bits]\n", argv[0]);
    return 1;
}
