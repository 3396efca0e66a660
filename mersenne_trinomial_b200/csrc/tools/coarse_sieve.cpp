// coarse_sieve -- drop-in for the reference's coarse_sieve tool
// (coarse_sieve.cu main, 1273-1570) on the B200 engine (libgf2e.so).
//
//   coarse_sieve <r> <depth> <out_prefix> [--smax S] [--found] [--cert|--no-cert]
//                [--no-survivors] [--load f.found.bin] [--load-survivors f]
//                [--min-depth D] [--checkpoint f] [--checkpoint-mins N]
//                [--checkpoint-keep G] [--resume f] [--gpus N]
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
// GF2E_SIEVE_WIDE_GB, default 64 GB: one slice up to d = 33).
//
// Checkpoints (coarse_sieve.cu:509-831, 1383-1480) use the reference's file
// layout (sieve_ckpt.h), so a stopped run resumes under either tool.  With
// --checkpoint the degrees run one library call each; best[] is saved at
// degree boundaries every --checkpoint-mins minutes and on SIGTERM/SIGINT,
// which stop the run with exit status 0.  A stop is honoured when the
// current degree ends; during degrees of 36 and up (seconds to minutes at
// r = 136279841) a watcher thread saves the last boundary at once instead.
// --resume continues from a checkpoint (into the same file unless
// --checkpoint names another); COARSE_TEST_STOP_AFTER_BUCKETS=N stops after
// N completed degrees, the reference's deterministic test hook with a
// degree as this engine's unit of resumable work.
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <chrono>
#include <csignal>
#include <mutex>
#include <string>
#include <thread>
#include <unistd.h>
#include <vector>

#include "certfmt.h"
#include "gf2e.h"
#include "sieve_ckpt.h"

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

// Checkpointing state of this run.  The signal handler only sets `stop`;
// files are written by the main thread between degrees, or by the watcher
// thread while a long degree is on the device.
struct CkptRun {
    bool on = false;
    std::string path;
    int keep = 3;
    double period_s = 0, last_write = 0;
    u64 r = 0, smax = 0;
    int depth = 0;
    sieve_ckpt::Baseline base;
    long stop_after = 0, degrees_done = 0;   // COARSE_TEST_STOP_AFTER_BUCKETS
    std::atomic<int> stop{0};                // set by the signal handler (lock-free)
    std::mutex mu;                           // guards snap / snap_pt
    std::vector<u64> snap;                   // best[] at snap_pt
    sieve_ckpt::Point snap_pt;
    bool snap_valid = false;
    std::atomic<bool> long_degree{false};    // the watcher may write for us
    std::atomic<bool> writer_claimed{false}; // one final write, by one thread
    std::atomic<bool> done{false};
};
static CkptRun g_ck;

static_assert(std::atomic<int>::is_always_lock_free, "the stop flag is set in a signal handler");
extern "C" void ckpt_on_signal(int) { g_ck.stop.store(1); }

// degrees from here on take seconds to minutes at full smax (d = 36: 4.5 s,
// d = 38: 151 s at r = 136279841), too long to wait for before saving
constexpr int kLongDegree = 36;

// write g_ck.snap (caller holds g_ck.mu)
static void ckpt_write_snapshot() {
    sieve_ckpt::WriteInfo info;
    const double t0 = now_s();
    if (!sieve_ckpt::write(g_ck.path, g_ck.keep, g_ck.r, g_ck.smax, g_ck.depth, g_ck.period_s,
                           g_ck.snap_pt, g_ck.snap, g_ck.base, &info))
        return;
    g_ck.last_write = now_s();
    if (info.delta)
        fprintf(stderr, "[checkpoint: d=%d, delta %" PRIu64 " entries (%.2f MB) -> %s, %.2fs]\n",
                g_ck.snap_pt.d, info.entries, info.bytes / 1048576.0, g_ck.path.c_str(),
                now_s() - t0);
    else
        fprintf(stderr, "[checkpoint: d=%d, full image (%.0f MB) -> %s, %.2fs]\n", g_ck.snap_pt.d,
                info.bytes / 1048576.0, g_ck.path.c_str(), now_s() - t0);
}

// host copy of best[] as the state "every degree below next_d is done"
static void ckpt_take(const u64 *dbest, int next_d) {
    std::lock_guard<std::mutex> lk(g_ck.mu);
    g_ck.snap.resize(g_ck.smax + 1);
    die_on(gf2e_copy_to_host(g_ck.snap.data(), dbest, (g_ck.smax + 1) * 8, nullptr), "snapshot");
    g_ck.snap_pt = sieve_ckpt::Point();
    g_ck.snap_pt.d = next_d;
    g_ck.snap_valid = true;
}

static void ckpt_stop_message() {
    fprintf(stderr, "stopping on request; resume with --resume %s\n", g_ck.path.c_str());
}

// Saves the last degree boundary when a stop arrives during a long degree,
// then ends the process (the degree in flight is abandoned and runs again
// on resume).
static void ckpt_watcher() {
    while (!g_ck.done.load()) {
        if (g_ck.stop.load() && g_ck.long_degree.load() && !g_ck.writer_claimed.exchange(true)) {
            {
                std::lock_guard<std::mutex> lk(g_ck.mu);
                if (g_ck.snap_valid) ckpt_write_snapshot();
            }
            ckpt_stop_message();
            fflush(stderr);
            _exit(0);
        }
        std::this_thread::sleep_for(std::chrono::milliseconds(100));
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
    u64 classes[41] = {0}, marks[41] = {0};
    const double t0 = now_s();
    if (min_depth > depth) {
        // resumed after the last degree: nothing left but the outputs
    } else if (!g_ck.on) {
        die_on(gf2e_sieve_run(r, min_depth, depth, smax, (u64 *)dbest, ws, ws_bytes, nullptr),
               "sieve");
        die_on(gf2e_sieve_stats(ws, depth, classes, marks, nullptr), "stats");
    } else {
        std::thread watcher(ckpt_watcher);
        for (int d = min_depth; d <= depth; d++) {
            if (d >= kLongDegree) {
                ckpt_take((const u64 *)dbest, d);       // what the watcher would save
                g_ck.long_degree = true;
            }
            die_on(gf2e_sieve_run(r, d, d, smax, (u64 *)dbest, ws, ws_bytes, nullptr), "sieve");
            g_ck.long_degree = false;
            u64 c[41] = {0}, m[41] = {0};
            die_on(gf2e_sieve_stats(ws, depth, c, m, nullptr), "stats");
            classes[d] = c[d];
            marks[d] = m[d];
            g_ck.degrees_done++;
            const bool test_stop = g_ck.stop_after > 0 && g_ck.degrees_done >= g_ck.stop_after;
            if ((g_ck.stop.load() || test_stop) && d < depth) {
                if (g_ck.writer_claimed.exchange(true))   // the watcher is saving and exiting
                    for (;;) pause();
                ckpt_take((const u64 *)dbest, d + 1);
                {
                    std::lock_guard<std::mutex> lk(g_ck.mu);
                    ckpt_write_snapshot();
                }
                ckpt_stop_message();
                fflush(nullptr);
                _exit(0);     // the watcher thread still runs: no static destructors
            }
            if (d < depth && g_ck.period_s > 0 && now_s() - g_ck.last_write >= g_ck.period_s) {
                ckpt_take((const u64 *)dbest, d + 1);
                std::lock_guard<std::mutex> lk(g_ck.mu);
                ckpt_write_snapshot();
            }
        }
        g_ck.done = true;
        watcher.join();
    }
    const double t1 = now_s();
    for (int d = min_depth; d <= depth; d++)
        fprintf(stderr, "d=%2d done: %" PRIu64 " classes, %" PRIu64 " marks\n", d, classes[d],
                marks[d]);
    fprintf(stderr, "device sieve time (degrees %d..%d): %.4fs\n", min_depth, depth, t1 - t0);
    best.resize(smax + 1);
    die_on(gf2e_copy_to_host(best.data(), dbest, (smax + 1) * 8, nullptr), "download");
    gf2e_device_free(ws);
    gf2e_device_free(dbest);
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
                        "         --load f.found.bin --load-survivors f --min-depth D --gpus N\n"
                        "         --checkpoint f --checkpoint-mins N --checkpoint-keep G "
                        "--resume f\n",
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
    const char *ckpt_path = nullptr, *resume_path = nullptr;
    double ckpt_mins = -1;                       // < 0: not given
    int ckpt_keep = 3;
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
        else if (!strcmp(argv[a], "--checkpoint") && a + 1 < argc) ckpt_path = argv[++a];
        else if (!strcmp(argv[a], "--checkpoint-mins") && a + 1 < argc) ckpt_mins = atof(argv[++a]);
        else if (!strcmp(argv[a], "--checkpoint-keep") && a + 1 < argc) ckpt_keep = atoi(argv[++a]);
        else if (!strcmp(argv[a], "--resume") && a + 1 < argc) resume_path = argv[++a];
        else if (!strcmp(argv[a], "--gpus") && a + 1 < argc) {
            fprintf(stderr, "note: --gpus %s ignored (this tool drives one GPU)\n", argv[a + 1]);
            a++;
        } else fprintf(stderr, "warning: ignoring unknown argument '%s'\n", argv[a]);
    }
    if (min_depth < 2) min_depth = 2;
    if (depth > 40) {
        fprintf(stderr, "depth %d > 40 is not supported by this engine\n", depth);
        return 1;
    }
    if (ckpt_keep < 1) ckpt_keep = 1;
    if (const char *e = getenv("COARSE_TEST_STOP_AFTER_BUCKETS")) g_ck.stop_after = atol(e);
    std::vector<u64> preload;
    const std::vector<u64> *pre = nullptr;
    double stored_period_s = 0;
    if (resume_path) {
        sieve_ckpt::Point pt;
        std::string used;
        if (!sieve_ckpt::read(resume_path, r, smax, preload, pt, stored_period_s, g_ck.base, &used))
            return 1;
        pre = &preload;
        min_depth = pt.d;
        u64 open = 0;
        for (u64 s = 1; s <= smax; s++) open += preload[s] == ~0ULL;
        if (pt.next > 0)
            fprintf(stderr, "note: %s stopped inside degree %d (bucket %d/%d); degree %d runs "
                            "again whole\n", used.c_str(), pt.d, pt.next, pt.nbuckets, pt.d);
        fprintf(stderr, "resumed %s: %" PRIu64 " survivors carried in; continuing at degree %d, "
                        "up to depth %d\n", used.c_str(), open, min_depth, depth);
        if (min_depth < 2) min_depth = 2;
    } else if (load_path) {
        if (!sieve_ckpt::load_found(load_path, smax, preload)) return 1;
        pre = &preload;
        g_ck.base.kind = 1;                       // baseline of delta checkpoints
        g_ck.base.path = load_path;
        g_ck.base.image = preload;
        g_ck.base.hash = sieve_ckpt::image_hash(preload.data() + 1, smax);
    } else if (loadsurv) {
        u64 listed = 0, oor = 0;
        if (!sieve_ckpt::load_survivors(loadsurv, smax, preload, &listed, &oor)) return 1;
        if (oor)
            fprintf(stderr, "warning: %" PRIu64 " survivor entries outside 1..%" PRIu64
                            " ignored\n", oor, smax);
        pre = &preload;
        g_ck.base.kind = 2;
        g_ck.base.path = loadsurv;
        g_ck.base.image = preload;
        g_ck.base.hash = sieve_ckpt::image_hash(preload.data() + 1, smax);
    } else if (min_depth > 2) {
        fprintf(stderr, "warning: --min-depth %d without --load means degrees 2..%d are not "
                        "computed\n", min_depth, min_depth - 1);
    }
    if (resume_path && !ckpt_path) ckpt_path = resume_path;   // keep saving to the same file
    if (ckpt_path) {
        g_ck.on = true;
        g_ck.path = ckpt_path;
        g_ck.keep = ckpt_keep;
        g_ck.period_s = ckpt_mins >= 0 ? ckpt_mins * 60.0 : stored_period_s;
        g_ck.last_write = now_s();
        g_ck.r = r;
        g_ck.smax = smax;
        g_ck.depth = depth;
        struct sigaction sa;
        memset(&sa, 0, sizeof sa);
        sa.sa_handler = ckpt_on_signal;
        sigaction(SIGTERM, &sa, nullptr);
        sigaction(SIGINT, &sa, nullptr);
        fprintf(stderr, "checkpointing to %s (%s, keeping %d generation%s)", ckpt_path,
                g_ck.base.usable(smax) ? "delta vs baseline" : "full image", g_ck.keep,
                g_ck.keep == 1 ? "" : "s");
        if (g_ck.period_s > 0) fprintf(stderr, ", every %.1f min", g_ck.period_s / 60.0);
        fprintf(stderr, "; SIGTERM/SIGINT saves and exits\n");
    }
    if (min_depth > depth) {
        fprintf(stderr, "nothing to sieve: degrees up to %d are already done\n", depth);
        min_depth = depth + 1;
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
        const bool ok = certfmt::write_lines(fs, best.data() + 1, smax, 1,
                                             certfmt::Lines::Survivors) >= 0;
        if (fclose(fs) != 0 || !ok) { fprintf(stderr, "%s: write failed\n", path); return 1; }
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
        const long long nc = certfmt::write_lines(fc, best.data() + 1, smax, 1,
                                                  certfmt::Lines::Cert);
        if (fclose(fc) != 0 || nc < 0) { fprintf(stderr, "%s: write failed\n", path); return 1; }
        fprintf(stderr, "%lld factors -> %s\n", nc, path);
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
