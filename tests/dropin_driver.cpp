// dropin_driver.cpp -- a translation unit written against the drop-in
// headers the way the reference's own tools use gf2_cantor_engine.h,
// gf2_cantor_cuda.h and gf2_trinomial_cuda.h (e.g. tsfactor.cu:1957-2006:
// G.F.n, G.dFA, G.F.fwd, k_pack, k_pointwise, k_overlap_add), driven by
// tests/test_gpu_dropin.py, which checks every output file against the
// oracle.  Inputs and outputs are raw little-endian u64 files.
//
//   dropin_driver fft <m> <in> <out>            CantorFFT fwd -> out, inv -> out.inv
//   dropin_driver twiddles <m> <out>            CantorFFT::W -> out, CudaFFT::dW -> out.dW
//   dropin_driver mulbuf <ab> <bb> <a> <b> <out> gf2x_fft_mul_buf (+ out.FA, out.FB)
//   dropin_driver naive|comb <ab> <bb> <a> <b> <out>
//   dropin_driver modp <d> <seed> <a> <abits>   prints "q residue"
//   dropin_driver trin <r> <s> <k> <out>        TrinGPU: F_k -> out, F_{k+1} through
//                                               G.F / dFA / dFB -> out.fft, through
//                                               square_A -> out.sq, cpu_square_mod ->
//                                               out.cpu, F_k * F_k mod T by
//                                               cpu_mod_trinomial -> out.mod
#include <cinttypes>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "gf2e_trinomial.hpp"

static std::vector<u64> load(const char *path) {
    std::vector<u64> v;
    FILE *f = fopen(path, "rb");
    if (!f) { perror(path); exit(2); }
    u64 w;
    while (fread(&w, 8, 1, f) == 1) v.push_back(w);
    fclose(f);
    return v;
}

static void save(const std::string &path, const u64 *p, size_t n) {
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) { perror(path.c_str()); exit(2); }
    fwrite(p, 8, n, f);
    fclose(f);
}

static std::vector<u64> read_dev(const u64 *d, size_t n) {
    std::vector<u64> h(n);
    gf2e_or_die(gf2e_copy_to_host(h.data(), d, n * 8, nullptr), "readback");
    return h;
}

int main(int argc, char **argv) {
    if (argc < 2) return 2;
    const std::string cmd = argv[1];
    CantorBasis B;
    B.build();
    if (cmd == "fft" && argc == 5) {
        const int m = atoi(argv[2]);
        std::vector<u64> f = load(argv[3]);
        CantorFFT F;
        F.init(m, B);
        if (f.size() != F.n) return 2;
        F.fwd(f.data());
        save(argv[4], f.data(), F.n);
        F.inv(f.data());
        save(std::string(argv[4]) + ".inv", f.data(), F.n);
        return 0;
    }
    if (cmd == "twiddles" && argc == 4) {
        const int m = atoi(argv[2]);
        CantorFFT F;
        F.init(m, B);
        save(argv[3], F.W.data(), F.W.size());
        CudaFFT G;
        G.init(m, B);
        std::vector<u64> dw = read_dev(G.dW, G.n / 2);
        save(std::string(argv[3]) + ".dW", dw.data(), dw.size());
        G.fini();
        return 0;
    }
    if ((cmd == "mulbuf" || cmd == "naive" || cmd == "comb") && argc == 7) {
        const u64 ab = strtoull(argv[2], 0, 10), bb = strtoull(argv[3], 0, 10);
        std::vector<u64> a = load(argv[4]), b = load(argv[5]);
        std::vector<u64> out(mul_out_words(ab, bb));
        if (cmd == "mulbuf") {
            CantorFFT F;
            F.init(gf2e_mul_fft_m(ab, bb), B);
            std::vector<u64> FA(F.n), FB(F.n);
            gf2x_fft_mul_buf(a.data(), ab, b.data(), bb, out.data(), F, FA.data(), FB.data());
            save(std::string(argv[6]) + ".FA", FA.data(), F.n);
            save(std::string(argv[6]) + ".FB", FB.data(), F.n);
        } else if (cmd == "naive") {
            gf2x_naive_mul(a.data(), ab, b.data(), bb, out.data());
        } else {
            gf2x_comb_mul(a.data(), ab, b.data(), bb, out.data());
        }
        save(argv[6], out.data(), out.size());
        return 0;
    }
    if (cmd == "modp" && argc == 6) {
        ModP p = find_irreducible_modp(atoi(argv[2]), strtoull(argv[3], 0, 0));
        std::vector<u64> a = load(argv[4]);
        printf("%" PRIu64 " %" PRIu64 "\n", p.q, p.residue(a.data(), strtoull(argv[5], 0, 10)));
        return 0;
    }
    if (cmd == "trin" && argc == 6) {
        const u64 r = strtoull(argv[2], 0, 10), s = strtoull(argv[3], 0, 10);
        const int k = atoi(argv[4]);
        const std::string out = argv[5];
        TrinGPU G;
        G.init(r);
        G.set_s(s);
        if (G.m != gf2e_mul_fft_m(r, r) || G.F.n != ((size_t)1 << G.m) || !G.dT1 || !G.dFA ||
            !G.dFB || G.nw2 != 2 * G.nw) {
            fprintf(stderr, "TrinGPU members\n");
            return 1;
        }
        gf2e_or_die(gf2e_trin_set_x(G.dA, G.nw, 1, r, nullptr), "set x");
        for (int i = 0; i < k; i++) G.square_A();
        std::vector<u64> fk = read_dev(G.dA, G.nw);
        save(out, fk.data(), G.nw);
        // F_k^2 by the product path of the reference's modmul breakdown
        const size_t ca = (size_t)((r + 31) >> 5);
        k_pack(G.dA, G.nw, G.dFA, ca, G.F.n);
        k_pack(G.dA, G.nw, G.dFB, ca, G.F.n);
        G.F.fwd(G.dFA);
        G.F.fwd(G.dFB);
        k_pointwise(G.dFA, G.dFB, G.F.n);
        G.F.inv(G.dFA);
        k_overlap_add(G.dFA, 2 * ca - 1, G.dT0, G.nw2);
        G.reduce(G.dT1, 2 * r - 1);
        std::vector<u64> v = read_dev(G.dT1, G.nw);
        save(out + ".fft", v.data(), G.nw);
        G.square_A();
        v = read_dev(G.dA, G.nw);
        save(out + ".sq", v.data(), G.nw);
        std::vector<u64> c = fk;
        cpu_square_mod(c, r, s);
        save(out + ".cpu", c.data(), c.size());
        // F_k * F_k as a 2r-1 bit product, folded by cpu_mod_trinomial
        std::vector<u64> prod(mul_out_words(r, r));
        gf2x_fft_mul(fk.data(), r, fk.data(), r, prod.data(), G.Bb);
        cpu_mod_trinomial(prod, 2 * r - 1, r, s);
        save(out + ".mod", prod.data(), G.nw);
        G.fini();
        return 0;
    }
    fprintf(stderr, "bad command\n");
    return 2;
}
