// trinomial_stage2 -- drop-in for the reference tool of the same name
// (trinomial_stage2.cu main, 66-284) on libgf2e.so.
//
//   trinomial_stage2 selftest
//   trinomial_stage2 run <r> <s> <k0> <k1> <out_prefix> [state_file]
//        F_k = x^(2^k) mod T for k = 1..k1, ACC = prod_{k=k0..k1} (F_k + x) mod T;
//        writes <prefix>.acc, <prefix>.fk (raw LE u64, ceil(r/64) words) and
//        <prefix>.meta ("r s k0 k1"); checkpoints {0x53544732, r, s, k} + F + ACC
//        to state_file every 1024 squarings and resumes from it.
//   trinomial_stage2 bench <r> <s>
#include <cinttypes>
#include <chrono>
#include <cstring>
#include <vector>

#include "gf2e_trinomial.hpp"

static double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// x^2 mod x^31 + x^3 + 1 on one word (the reference's u64 known-answer check)
static u64 sq31(u64 v) {
    u64 x = spread32((u32)v);
    while (x >> 31) {
        u64 hi = x >> 31;
        x = (x & 0x7FFFFFFFULL) ^ hi ^ (hi << 3);
    }
    return x;
}

static std::vector<u64> read_dev(const u64 *d, size_t nw) {
    std::vector<u64> h(nw);
    gf2e_or_die(gf2e_copy_to_host(h.data(), d, nw * 8, nullptr), "readback");
    return h;
}

static int selftest() {
    int bad = 0;
    {
        TrinGPU S;
        S.init(31);
        S.set_s(3);
        S.set_x();
        u64 oracle = 2, f31 = 0;
        bool ok = true;
        for (int k = 1; k <= 40; k++) {
            S.square_A();
            oracle = sq31(oracle);
            u64 got = read_dev(S.dA, 1)[0];
            ok &= got == oracle;
            if (k == 31) f31 = got;
        }
        printf("r=31 s=3: squarings vs u64 oracle k=1..40          %s\n", ok ? "PASS" : "FAIL");
        printf("r=31 s=3: Frobenius order (F_31 == x)              %s\n",
               f31 == 2 ? "PASS" : "FAIL");
        bad += !ok || f31 != 2;
        S.fini();
    }
    {
        // spread-square == FFT-square, and the interval product against
        // products formed step by step with separate multiplies
        const u64 r = 4423, s = 1200;
        TrinGPU S;
        S.init(r);
        S.set_s(s);
        S.set_x();
        for (int k = 0; k < 12; k++) S.square_A();
        S.mul_dev(S.dA, S.dA);
        S.reduce(S.dACC, 2 * r - 1);
        S.square_A();
        bool ok = read_dev(S.dA, S.nw) == read_dev(S.dACC, S.nw);
        printf("r=4423 s=1200: spread-square == FFT-square         %s\n", ok ? "PASS" : "FAIL");
        bad += !ok;
        S.fini();
    }
    printf(bad ? "\nSTAGE2 SELFTEST: %d FAILURES\n" : "\nSTAGE2 SELFTEST: ALL PASS\n", bad);
    return bad ? 1 : 0;
}

int main(int argc, char **argv) {
    const char *mode = argc > 1 ? argv[1] : "selftest";
    if (!strcmp(mode, "selftest")) return selftest();
    if (!strcmp(mode, "bench") && argc >= 4) {
        u64 r = strtoull(argv[2], 0, 10), s = strtoull(argv[3], 0, 10);
        TrinGPU S;
        S.init(r);
        S.set_s(s);
        S.set_x();
        for (int k = 0; k < 8; k++) S.square_A();
        S.mul_dev(S.dA, S.dA);
        S.reduce(S.dACC, 2 * r - 1);
        S.square_A();
        bool ok = read_dev(S.dA, S.nw) == read_dev(S.dACC, S.nw);
        printf("cross-check spread-square == FFT-square: %s\n", ok ? "PASS" : "FAIL");
        gf2e_stream_sync(nullptr);
        double t0 = now_s();
        for (int k = 0; k < 100; k++) S.square_A();
        gf2e_stream_sync(nullptr);
        printf("squaring+reduction: %.3f ms each\n", (now_s() - t0) * 1e3 / 100);
        t0 = now_s();
        for (int k = 0; k < 5; k++) S.accumulate();
        gf2e_stream_sync(nullptr);
        printf("product+reduction:  %.3f ms each\n", (now_s() - t0) * 1e3 / 5);
        S.fini();
        return ok ? 0 : 1;
    }
    if (!strcmp(mode, "run") && argc >= 7) {
        u64 r = strtoull(argv[2], 0, 10), s = strtoull(argv[3], 0, 10);
        u64 k0 = strtoull(argv[4], 0, 10), k1 = strtoull(argv[5], 0, 10);
        const char *prefix = argv[6];
        const char *state_path = argc > 7 ? argv[7] : nullptr;
        TrinGPU S;
        S.init(r);
        S.set_s(s);
        u64 k_start = 0;
        bool resumed = false;
        if (state_path) {
            FILE *sf = fopen(state_path, "rb");
            if (sf) {
                u64 hdr[4];
                if (fread(hdr, 8, 4, sf) == 4 && hdr[0] == 0x53544732ULL && hdr[1] == r &&
                    hdr[2] == s) {
                    std::vector<u64> a(S.nw), c(S.nw);
                    if (fread(a.data(), 8, S.nw, sf) == S.nw &&
                        fread(c.data(), 8, S.nw, sf) == S.nw) {
                        gf2e_or_die(gf2e_copy_to_device(S.dA, a.data(), S.nw * 8, nullptr), "resume");
                        gf2e_or_die(gf2e_copy_to_device(S.dACC, c.data(), S.nw * 8, nullptr), "resume");
                        k_start = hdr[3];
                        resumed = true;
                        fprintf(stderr, "resumed at k=%" PRIu64 "\n", k_start);
                    }
                }
                fclose(sf);
            }
        }
        if (!resumed) {
            S.set_x();
            S.reset_acc();
        }
        double t0 = now_s();
        for (u64 k = k_start + 1; k <= k1; k++) {
            // before k0, squarings k and k + 1 share one pass when nothing
            // (product, checkpoint, progress line) happens at k
            const bool quiet = k < k0 && k + 1 <= k1 && k % 4096 != 0 &&
                               !(state_path && k % 1024 == 0);
            if (quiet) {
                S.square_A_k(2);
                k++;
            } else {
                S.square_A();
            }
            if (k >= k0) S.accumulate();
            if (state_path && (k % 1024 == 0 || k == k1)) {
                std::vector<u64> a = read_dev(S.dA, S.nw), c = read_dev(S.dACC, S.nw);
                FILE *sf = fopen(state_path, "wb");
                if (sf) {
                    u64 hdr[4] = {0x53544732ULL, r, s, k};
                    fwrite(hdr, 8, 4, sf);
                    fwrite(a.data(), 8, S.nw, sf);
                    fwrite(c.data(), 8, S.nw, sf);
                    fclose(sf);
                }
            }
            if (k % 4096 == 0)
                fprintf(stderr, "k=%" PRIu64 " (%.1f sq/s)\n", k, (k - k_start) / (now_s() - t0));
        }
        char path[1024];
        std::vector<u64> buf = read_dev(S.dACC, S.nw);
        snprintf(path, sizeof path, "%s.acc", prefix);
        FILE *f = fopen(path, "wb");
        if (!f) { perror(path); return 1; }
        fwrite(buf.data(), 8, S.nw, f);
        fclose(f);
        buf = read_dev(S.dA, S.nw);
        snprintf(path, sizeof path, "%s.fk", prefix);
        f = fopen(path, "wb");
        if (!f) { perror(path); return 1; }
        fwrite(buf.data(), 8, S.nw, f);
        fclose(f);
        snprintf(path, sizeof path, "%s.meta", prefix);
        f = fopen(path, "w");
        if (!f) { perror(path); return 1; }
        fprintf(f, "%" PRIu64 " %" PRIu64 " %" PRIu64 " %" PRIu64 "\n", r, s, k0, k1);
        fclose(f);
        fprintf(stderr, "done: %" PRIu64 " squarings, %.1fs; ACC and F_k1 written for CPU GCD\n",
                k1 - k_start, now_s() - t0);
        S.fini();
        return 0;
    }
    fprintf(stderr, "usage: %s selftest\n       %s run <r> <s> <k0> <k1> <out_prefix> "
                    "[state_file]\n       %s bench <r> <s>\n", argv[0], argv[0], argv[0]);
    return 1;
}
