// Test driver for the sieve checkpoint files (mersenne_trinomial_b200/csrc/
// tools/sieve_ckpt.h), compiled by tests/test_sieve_ckpt.py.  Host only.
//
//   ckpt_driver write <path> <keep> <r> <smax> <depth> <period_s> <d> <next> <nbuckets>
//                     <keys.bin> [<baseline kind 1|2> <baseline path>]
//   ckpt_driver read  <path> <r> <smax> <keys_out.bin>
//
// keys files hold smax LE u64 keys for s = 1..smax (the .found.bin layout).
// `write` prints "delta <0|1> entries <n> bytes <b>"; `read` prints
// "d <d> next <n> nbuckets <nb> period <p> used <file> base <kind>".
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "sieve_ckpt.h"

using sieve_ckpt::u64;

static bool load_keys(const char *path, u64 smax, std::vector<u64> &v) {
    return sieve_ckpt::load_found(path, smax, v);
}

int main(int argc, char **argv) {
    if (argc >= 12 && !strcmp(argv[1], "write")) {
        const std::string path = argv[2];
        const int keep = atoi(argv[3]);
        const u64 r = strtoull(argv[4], 0, 10), smax = strtoull(argv[5], 0, 10);
        const int depth = atoi(argv[6]);
        const double period = atof(argv[7]);
        sieve_ckpt::Point pt;
        pt.d = atoi(argv[8]);
        pt.next = atoi(argv[9]);
        pt.nbuckets = atoi(argv[10]);
        std::vector<u64> best;
        if (!load_keys(argv[11], smax, best)) return 2;
        sieve_ckpt::Baseline base;
        if (argc >= 14) {
            base.kind = atoi(argv[12]);
            base.path = argv[13];
            if (!sieve_ckpt::load_baseline(base, smax)) return 2;
            base.hash = sieve_ckpt::image_hash(base.image.data() + 1, smax);
        }
        sieve_ckpt::WriteInfo info;
        if (!sieve_ckpt::write(path, keep, r, smax, depth, period, pt, best, base, &info)) return 1;
        printf("delta %d entries %" PRIu64 " bytes %" PRIu64 "\n", info.delta ? 1 : 0, info.entries,
               info.bytes);
        return 0;
    }
    if (argc >= 6 && !strcmp(argv[1], "read")) {
        const u64 r = strtoull(argv[3], 0, 10), smax = strtoull(argv[4], 0, 10);
        std::vector<u64> best;
        sieve_ckpt::Point pt;
        sieve_ckpt::Baseline base;
        double period = 0;
        std::string used;
        if (!sieve_ckpt::read(argv[2], r, smax, best, pt, period, base, &used)) return 1;
        FILE *f = fopen(argv[5], "wb");
        if (!f || fwrite(best.data() + 1, 8, smax, f) != smax) return 2;
        fclose(f);
        printf("d %d next %d nbuckets %d period %.0f used %s base %d\n", pt.d, pt.next, pt.nbuckets,
               period, used.c_str(), base.kind);
        return 0;
    }
    fprintf(stderr, "usage: see the header of this file\n");
    return 2;
}
