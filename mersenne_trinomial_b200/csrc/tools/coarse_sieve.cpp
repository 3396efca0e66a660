// coarse_sieve -- drop-in for the reference's coarse_sieve tool
// (coarse_sieve.cu main, 1273-1570) on the B200 engine (libgf2e.so).
//
//   coarse_sieve <r> <depth> <out_prefix> [--smax S] [--found] [--cert|--no-cert]
//                [--no-survivors] [--load f.found.bin] [--load-survivors f]
//                [--min-depth D] [--gpus N]
//   coarse_sieve <r> <depth> <smax> <out_prefix> ...      (legacy positional form)
//   coarse_sieve --selftest
//
// Outputs (same formats as the reference, coarse_sieve.cu:1510-1558):
//   <prefix>.survivors.txt  s with no factor of degree <= depth, one per line
//   <prefix>.found.cert     "s d p<hex>" ascending s (default on)
//   <prefix>.found.bin      LE u64 key per s = 1..smax, UINT64_MAX = none (--found)
// Degrees up to 31 run on dense tables in HBM (the reference needs its
// bucketed low-memory mode beyond d = 29 on an 8 GB GPU); degrees 32..40 on
// the wide path (64-bit elements, the log table in slices of at most
// GF2E_SIEVE_WIDE_GB, default 64 GB: one slice up to d = 33).  Checkpoint
// flags (--checkpoint, --checkpoint-mins, --checkpoint-keep, --resume) are
// accepted and ignored with a note.
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <chrono>
#include <string>
#include <vector>

#include "gf2e.h"

typedef uint64_t u64;

static double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

static void die_on(int st, const char *what) {
    if (st != GF2E_OK) {
        fprintf(stderr, "%s: %s (%s)\n", what, gf2e_status_string(st), gf2e_last_error());
        exit(1);
    }
}

// run the sieve on the device; best has smax+1 entries (index 0 unused)
static void run_gpu(u64 r, int depth, u64 smax, int min_depth, std::vector<u64> &best,
                    const std::vector<u64> *preload) {
    size_t ws_bytes = 0;
    die_on(gf2e_sieve_workspace_size(depth, &ws_bytes), "workspace");
    void *ws = nullptr, *dbest = nullptr;
    die_on(gf2e_device_alloc(&ws, ws_bytes), "alloc workspace");
    die_on(gf2e_device_alloc(&dbest, (smax + 1) * 8), "alloc best");
    if (preload)
        die_on(gf2e_copy_to_device(dbest, preload->data(), (smax + 1) * 8, nullptr), "upload");
    else
        die_on(gf2e_sieve_fill((u64 *)dbest, smax, nullptr), "fill");
    double t0 = now_s();
    die_on(gf2e_sieve_run(r, min_depth, depth, smax, (u64 *)dbest, ws, ws_bytes, nullptr),
           "sieve");
    double t1 = now_s();
    u64 classes[41], marks[41];
    die_on(gf2e_sieve_stats(ws, depth, classes, marks, nullptr), "stats");
    for (int d = min_depth; d <= depth; d++)
        fprintf(stderr, "d=%2d done: %" PRIu64 " classes, %" PRIu64 " marks\n", d, classes[d],
                marks[d]);
    fprintf(stderr, "device sieve time (degrees %d..%d): %.4fs\n", min_depth, depth, t1 - t0);
    best.resize(smax + 1);
    die_on(gf2e_copy_to_host(best.data(), dbest, (smax + 1) * 8, nullptr), "download");
    gf2e_device_free(ws);
    gf2e_device_free(dbest);
}

static bool read_found_image(const char *path, u64 smax, std::vector<u64> &out) {
    FILE *f = fopen(path, "rb");
    if (!f) { perror(path); return false; }
    out.assign(smax + 1, ~0ULL);
    size_t got = fread(out.data() + 1, 8, smax, f);
    fclose(f);
    if (got != smax) {
        fprintf(stderr, "%s: expected %" PRIu64 " keys, got %zu\n", path, smax, got);
        return false;
    }
    return true;
}

static bool read_survivors(const char *path, u64 smax, int min_depth, std::vector<u64> &out) {
    FILE *f = fopen(path, "r");
    if (!f) { perror(path); return false; }
    // every s not listed already has a factor of degree < min_depth; a
    // sentinel below (min_depth << 48) blocks all new marks exactly as the
    // real key would (coarse_sieve.cu:1466-1480)
    out.assign(smax + 1, 0);
    u64 s;
    while (fscanf(f, "%" SCNu64, &s) == 1)
        if (s >= 1 && s <= smax) out[s] = ~0ULL;
    fclose(f);
    (void)min_depth;
    return true;
}

static int selftest() {
    // GPU result checked two ways without a CPU sieve: (1) extending a
    // depth-12 run to depth 20 equals a direct depth-20 run, (2) every
    // reported factor divides its trinomial (check-ntl's test, on the host).
    const u64 r = 136279841, smax = 999999;
    printf("selftest: r=%" PRIu64 " depth=20 smax=%" PRIu64 "\n", r, smax);
    std::vector<u64> a, b, lo;
    run_gpu(r, 20, smax, 2, a, nullptr);
    run_gpu(r, 12, smax, 2, lo, nullptr);
    run_gpu(r, 20, smax, 13, b, &lo);
    u64 bad = 0, nf = 0;
    for (u64 s = 1; s <= smax; s++)
        if (a[s] != b[s] && ++bad <= 10)
            fprintf(stderr, "MISMATCH s=%" PRIu64 "\n", s);
    // divisibility: x^r + x^s + 1 == 0 mod p for the reported p (d <= 20 here)
    for (u64 s = 1; s <= smax; s++) {
        if (a[s] == ~0ULL) continue;
        nf++;
        int d = (int)(a[s] >> 48);
        u64 p = a[s] & 0xFFFFFFFFFFFFULL;
        auto mulmod = [&](u64 x, u64 y) {
            u64 acc = 0;
            for (int i = 0; i < d; i++)
                if ((y >> i) & 1) acc ^= x << i;
            for (int bit = 2 * d - 2; bit >= d; bit--)
                if ((acc >> bit) & 1) acc ^= p << (bit - d);
            return acc;
        };
        auto powx = [&](u64 e) {
            u64 res = 1, base = 2;
            if (d == 1) base = 0;
            while (e) { if (e & 1) res = mulmod(res, base); base = mulmod(base, base); e >>= 1; }
            return res;
        };
        if ((powx(r) ^ powx(s) ^ 1) != 0 && ++bad <= 10)
            fprintf(stderr, "NOT A FACTOR s=%" PRIu64 " d=%d p%" PRIx64 "\n", s, d, p);
    }
    printf("selftest: %" PRIu64 " factors checked: %s (%" PRIu64 " failures)\n", nf,
           bad ? "FAIL" : "PASS", bad);
    return bad ? 1 : 0;
}

int main(int argc, char **argv) {
    if (argc >= 2 && !strcmp(argv[1], "--selftest")) return selftest();
    if (argc >= 2 && !strcmp(argv[1], "--selftest-lowmem")) {
        fprintf(stderr, "note: degrees <= 31 use dense tables, 32..40 sliced log tables; "
                        "running the standard selftest\n");
        return selftest();
    }
    if (argc < 4) {
        fprintf(stderr, "usage: %s <r> <depth> <out_prefix> [options]\n"
                        "       %s --selftest\n"
                        "options: --smax S --found --cert --no-cert --no-survivors\n"
                        "         --load f.found.bin --load-survivors f --min-depth D --gpus N\n",
                argv[0], argv[0]);
        return 1;
    }
    u64 r = strtoull(argv[1], 0, 10);
    int depth = atoi(argv[2]);
    bool legacy = false;
    {
        const char *p = argv[3];
        bool alldig = *p != '\0';
        for (const char *c = p; *c; c++)
            if (*c < '0' || *c > '9') { alldig = false; break; }
        if (alldig && argc >= 5) legacy = true;
    }
    u64 smax = legacy ? strtoull(argv[3], 0, 10) : r / 2;
    const char *prefix = legacy ? argv[4] : argv[3];
    if (legacy)
        fprintf(stderr, "note: positional <smax> is deprecated; --smax <S> "
                        "(default floor(r/2) = %" PRIu64 ") is preferred\n", r / 2);
    bool write_found = false, write_surv = true, write_cert = true;
    const char *load_path = nullptr, *loadsurv = nullptr;
    int min_depth = 2;
    for (int a = legacy ? 5 : 4; a < argc; a++) {
        if (!strcmp(argv[a], "--found")) write_found = true;
        else if (!strcmp(argv[a], "--smax") && a + 1 < argc) smax = strtoull(argv[++a], 0, 10);
        else if (!strcmp(argv[a], "--cert")) write_cert = true;
        else if (!strcmp(argv[a], "--no-cert")) write_cert = false;
        else if (!strcmp(argv[a], "--no-survivors")) write_surv = false;
        else if (!strcmp(argv[a], "--load") && a + 1 < argc) load_path = argv[++a];
        else if (!strcmp(argv[a], "--load-survivors") && a + 1 < argc) loadsurv = argv[++a];
        else if (!strcmp(argv[a], "--min-depth") && a + 1 < argc) min_depth = atoi(argv[++a]);
        else if ((!strcmp(argv[a], "--checkpoint") || !strcmp(argv[a], "--checkpoint-mins") ||
                  !strcmp(argv[a], "--checkpoint-keep") || !strcmp(argv[a], "--resume") ||
                  !strcmp(argv[a], "--gpus")) && a + 1 < argc) {
            fprintf(stderr, "note: %s %s ignored (one GPU, no checkpoints)\n", argv[a],
                    argv[a + 1]);
            a++;
        } else fprintf(stderr, "warning: ignoring unknown argument '%s'\n", argv[a]);
    }
    if (min_depth < 2) min_depth = 2;
    if (depth > 40) {
        fprintf(stderr, "depth %d > 40 is not supported by this engine\n", depth);
        return 1;
    }
    std::vector<u64> preload;
    const std::vector<u64> *pre = nullptr;
    if (load_path) {
        if (!read_found_image(load_path, smax, preload)) return 1;
        pre = &preload;
    } else if (loadsurv) {
        if (!read_survivors(loadsurv, smax, min_depth, preload)) return 1;
        pre = &preload;
    } else if (min_depth > 2) {
        fprintf(stderr, "warning: --min-depth %d without --load means degrees 2..%d are not "
                        "computed\n", min_depth, min_depth - 1);
    }
    double t0 = now_s();
    std::vector<u64> best;
    run_gpu(r, depth, smax, min_depth, best, pre);
    fprintf(stderr, "total sieve time: %.2fs\n", now_s() - t0);

    char path[1024];
    u64 nsurv = 0;
    for (u64 s = 1; s <= smax; s++) nsurv += best[s] == ~0ULL;
    if (write_surv) {
        snprintf(path, sizeof path, "%s.survivors.txt", prefix);
        FILE *fs = fopen(path, "w");
        if (!fs) { perror(path); return 1; }
        for (u64 s = 1; s <= smax; s++)
            if (best[s] == ~0ULL) fprintf(fs, "%" PRIu64 "\n", s);
        fclose(fs);
        fprintf(stderr, "%" PRIu64 " survivors (no factor of degree <= %d) -> %s\n", nsurv,
                depth, path);
    } else {
        fprintf(stderr, "%" PRIu64 " survivors (no factor of degree <= %d) [survivors file "
                        "suppressed via --no-survivors]\n", nsurv, depth);
    }
    if (write_cert) {
        snprintf(path, sizeof path, "%s.found.cert", prefix);
        FILE *fc = fopen(path, "w");
        if (!fc) { perror(path); return 1; }
        u64 nc = 0;
        for (u64 s = 1; s <= smax; s++) {
            u64 b = best[s];
            if (b == ~0ULL || b == 0) continue;
            fprintf(fc, "%" PRIu64 " %u p%" PRIx64 "\n", s, (unsigned)(b >> 48),
                    b & 0xFFFFFFFFFFFFULL);
            nc++;
        }
        fclose(fc);
        fprintf(stderr, "%" PRIu64 " factors -> %s\n", nc, path);
    }
    if (write_found) {
        snprintf(path, sizeof path, "%s.found.bin", prefix);
        FILE *ff = fopen(path, "wb");
        if (!ff) { perror(path); return 1; }
        fwrite(best.data() + 1, 8, smax, ff);
        fclose(ff);
        fprintf(stderr, "packed keys for s=1..%" PRIu64 " -> %s\n", smax, path);
    }
    return 0;
}
