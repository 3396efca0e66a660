// trinomial_scan -- drop-in for the reference tool of the same name
// (trinomial_scan.cu main, 542-697) on libgf2e.so: the deep scan of sieve
// survivors, batched over the s values on the GPU with GPU gcds.
//
//   trinomial_scan <r> <survivors.txt> <k0> <maxd> <out_prefix>
//                  [--interval Lmax] [--l0 L0] [--batch B] [--block m] [--verbose 0..3]
//                  [--sched doubling|linear|opt] [--q0 N] [--sched-G N] [--sched-rho R]
//                  [--Zq N]                              (tsfactor's interval schedules)
//                  [--state FILE]                        (resume state, see below)
//                  [--gcd-threads N]                     (accepted, unused)
//   trinomial_scan --selftest
//
// Output <out_prefix>.results.txt, appended, resumable (s already listed are
// skipped): "s d p<hex>" (least degree, numerically least factor), "s u"
// (no factor of degree <= maxd) or "s rA-B" (a factor with degree in [A,B]
// that could not be isolated).  k0 must be the depth the sieve reached.
#include <cinttypes>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <vector>

#include "gf2e.h"

typedef uint64_t u64;

static double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

static std::string hexmask(const u64 *w, size_t n) {
    static const char *dig = "0123456789abcdef";
    long long d = -1;
    for (size_t i = n; i-- > 0;)
        if (w[i]) { d = (long long)(i * 64 + 63 - __builtin_clzll(w[i])); break; }
    if (d < 0) return "0";
    std::string s;
    for (long long k = d / 4; k >= 0; k--) s += dig[(w[k >> 4] >> ((k & 15) * 4)) & 0xF];
    return s;
}

// x^e mod p for a factor p of degree d (multi-word, shift-and-add)
static bool divides(u64 r, u64 s, const u64 *p, size_t pw, u64 d) {
    size_t nw = (size_t)(d / 64) + 1;
    std::vector<u64> P(p, p + pw);
    P.resize(nw + 1, 0);
    auto mulx_mod = [&](std::vector<u64> &a) {
        u64 carry = 0;
        for (size_t i = 0; i < nw; i++) { u64 nc = a[i] >> 63; a[i] = (a[i] << 1) | carry; carry = nc; }
        if ((a[d >> 6] >> (d & 63)) & 1)
            for (size_t i = 0; i < nw; i++) a[i] ^= P[i];
    };
    auto sqr_mod = [&](std::vector<u64> &a) {
        std::vector<u64> t(2 * nw + 1, 0);
        for (size_t i = 0; i < nw; i++)
            for (int b = 0; b < 64; b++)
                if ((a[i] >> b) & 1) {
                    u64 e = 2 * (i * 64 + b);
                    t[e >> 6] ^= 1ull << (e & 63);
                }
        for (long long e = (long long)(2 * nw * 64) - 1; e >= (long long)d; e--) {
            if (!((t[e >> 6] >> (e & 63)) & 1)) continue;
            u64 sh = (u64)e - d;
            for (size_t i = 0; i <= d / 64; i++) {
                u64 v = P[i];
                if (!v) continue;
                size_t j = i + (sh >> 6);
                unsigned bs = sh & 63;
                if (j < t.size()) t[j] ^= v << bs;
                if (bs && j + 1 < t.size()) t[j + 1] ^= v >> (64 - bs);
            }
        }
        for (size_t i = 0; i < nw; i++) a[i] = t[i];
    };
    auto powx = [&](u64 e) {
        std::vector<u64> a(nw, 0);
        a[0] = 1;
        for (int bit = 63; bit >= 0; bit--) {
            sqr_mod(a);
            if ((e >> bit) & 1) mulx_mod(a);
        }
        return a;
    };
    std::vector<u64> xr = powx(r), xs = powx(s);
    xr[0] ^= 1;
    for (size_t i = 0; i < nw; i++)
        if (xr[i] != xs[i]) return false;
    return true;
}

// Resume state (trinomial_scan.cu:144-170): records {0x4E435354, r, s, k, nw}
// followed by F_k = x^(2^k) mod T, k the verified frontier of an s in
// progress (every degree <= k clear).  The reference keeps one record, its
// one s in progress; this tool scans many s at once and writes one record
// per resident s, and reads every record of a file (a reference file is the
// one-record case).  Only k is needed to resume: the scan restarts that s
// at k0 = k, computing F_k again on the GPU.
static const u64 kStateMagic = 0x4E435354ULL;

static std::map<u64, u64> load_states(const char *path, u64 r, size_t nw) {
    std::map<u64, u64> out;
    FILE *f = path ? fopen(path, "rb") : nullptr;
    if (!f) return out;
    u64 hdr[5];
    std::vector<u64> F(nw);
    while (fread(hdr, 8, 5, f) == 5 && hdr[0] == kStateMagic && hdr[1] == r && hdr[4] == nw &&
           fread(F.data(), 8, nw, f) == nw)
        out[hdr[2]] = hdr[3];
    fclose(f);
    return out;
}

static bool save_states(const char *path, u64 r, size_t nw, const std::map<u64, u64> &fr) {
    std::string tmp = std::string(path) + ".tmp";
    FILE *f = fopen(tmp.c_str(), "wb");
    if (!f) return false;
    std::vector<u64> F(nw);
    bool ok = true;
    for (const auto &e : fr) {
        const u64 s = e.first, k = e.second;
        ok = gf2e_trin_frobenius_host(r, &s, 1, (uint32_t)k, F.data(), nw, nullptr) == GF2E_OK;
        if (!ok) break;
        const u64 hdr[5] = {kStateMagic, r, s, k, (u64)nw};
        ok = fwrite(hdr, 8, 5, f) == 5 && fwrite(F.data(), 8, nw, f) == nw;
        if (!ok) break;
    }
    ok = (fclose(f) == 0) && ok;
    if (ok) ok = rename(tmp.c_str(), path) == 0;
    return ok;
}

// Scan every s, writing each result line as soon as its s finishes (the
// reference appends per survivor too), with the resume state saved every
// 30 s (GF2E_SCAN_STATE_SECS) when a frontier moved.  `fres` null: results
// only counted.
static int run(u64 r, const std::vector<u64> &surv, u64 k0, u64 maxd, u64 L0, u64 Lmax,
               int batch, int block, const gf2e_sched &sched, FILE *fres, int verbose,
               const char *state_path, u64 *nfound, u64 *nu, u64 *nbad) {
    const size_t cap = 4096, nw = (size_t)((r + 63) >> 6);
    std::map<u64, u64> resume = load_states(state_path, r, nw);
    gf2e_scanner *S = nullptr;
    int st = gf2e_scanner_create_blocked(r, std::max(1, std::min<int>(batch, (int)surv.size())),
                                         block, &S);
    if (st == GF2E_OK) st = gf2e_scanner_set_schedule(S, &sched);
    auto fail = [&](int code) {
        fprintf(stderr, "scan failed: %s (%s)\n", gf2e_status_string(code), gf2e_last_error());
        if (S) gf2e_scanner_destroy(S);
        return 1;
    };
    if (st != GF2E_OK) return fail(st);
    size_t pending = 0;
    for (size_t i = 0; i < surv.size(); i++) {
        u64 start = k0;
        auto it = resume.find(surv[i]);
        if (it != resume.end() && it->second > k0) {
            start = std::min(it->second, maxd);
            if (verbose >= 1)
                fprintf(stderr, "  s=%" PRIu64 ": resumed at k=%" PRIu64 "\n", surv[i], start);
        }
        if (start >= maxd) {                            // nothing left below maxd
            if (fres) { fprintf(fres, "%" PRIu64 " u\n", surv[i]); fflush(fres); }
            ++*nu;
            continue;
        }
        st = gf2e_scanner_submit(S, &surv[i], 1, start, maxd, L0, Lmax, (u64)i);
        if (st != GF2E_OK) return fail(st);
        pending++;
    }
    std::vector<gf2e_scan_result> res(64);
    std::vector<u64> tags(64), masks(64 * cap);
    std::vector<u64> fs(batch), fk(batch);
    std::map<u64, u64> saved;
    double last_save = now_s(), save_every = 30.0;
    if (const char *e = getenv("GF2E_SCAN_STATE_SECS")) save_every = atof(e);
    while (pending > 0) {
        st = gf2e_scanner_step(S, 256, nullptr);
        if (st != GF2E_OK) return fail(st);
        int n = 0;
        do {
            st = gf2e_scanner_poll(S, res.data(), tags.data(), masks.data(), cap, 64, &n);
            if (st != GF2E_OK) return fail(st);
            for (int q = 0; q < n; q++) {
                const gf2e_scan_result &R = res[q];
                if (R.status == 1) {
                    std::string hx = hexmask(&masks[q * cap], R.mask_words);
                    if (fres) fprintf(fres, "%" PRIu64 " %" PRIu64 " p%s\n", R.s, R.d, hx.c_str());
                    if (!divides(r, R.s, &masks[q * cap], R.mask_words, R.d)) ++*nbad;
                    ++*nfound;
                    if (verbose >= 1) fprintf(stderr, "  s=%" PRIu64 ": d=%" PRIu64 "\n", R.s, R.d);
                } else if (R.status == 2) {
                    if (fres) fprintf(fres, "%" PRIu64 " u\n", R.s);
                    ++*nu;
                } else {
                    if (fres) fprintf(fres, "%" PRIu64 " r%" PRIu64 "-%" PRIu64 "\n", R.s, R.rlo, R.rhi);
                    ++*nfound;
                }
                pending--;
            }
            if (n && fres) fflush(fres);
        } while (n == 64);
        int q = 0, a = 0;
        gf2e_scanner_status(S, &q, &a, nullptr, nullptr);
        if (pending > 0 && q == 0 && a == 0) {
            fprintf(stderr, "scan failed: %zu results lost\n", pending);
            gf2e_scanner_destroy(S);
            return 1;
        }
        if (state_path && now_s() - last_save >= save_every) {
            int nf = 0;
            gf2e_scanner_frontiers(S, fs.data(), fk.data(), nullptr, batch, &nf);
            std::map<u64, u64> now;
            for (int i = 0; i < nf; i++)
                if (fk[i] > k0) now[fs[i]] = fk[i];
            if (!now.empty() && now != saved) {
                if (!save_states(state_path, r, nw, now))
                    fprintf(stderr, "warning: could not write state file %s\n", state_path);
                saved = now;
            }
            last_save = now_s();
        }
    }
    gf2e_scanner_destroy(S);
    return 0;
}

static int selftest() {
    // survivors of r = 4423 with no factor of degree <= 5 among s = 2..350
    const u64 r = 4423, k0 = 5, maxd = 200, smax = 350;
    size_t ws = 0;
    gf2e_sieve_workspace_size((int)k0, &ws);
    void *dws, *dbest;
    if (gf2e_device_alloc(&dws, ws) || gf2e_device_alloc(&dbest, 8 * (smax + 1))) return 1;
    gf2e_sieve_fill((u64 *)dbest, smax, nullptr);
    if (gf2e_sieve_run(r, 2, (int)k0, smax, (u64 *)dbest, dws, ws, nullptr) != GF2E_OK) return 1;
    std::vector<u64> best(smax + 1);
    gf2e_copy_to_host(best.data(), dbest, 8 * (smax + 1), nullptr);
    std::vector<u64> surv;
    for (u64 s = 2; s <= smax; s++)
        if (best[s] == ~0ULL) surv.push_back(s);
    int bad = 0;
    // interval policies: trinomial_scan's doubling, then tsfactor's blocked
    // DDF under its linear (m=4 q0=3) and Euler-optimal (m=6 G=60) schedules
    struct Pol { u64 L0, Lmax; int block; gf2e_sched sched; const char *name; };
    const Pol pol[] = {
        {32, 4096, 1, {GF2E_SCHED_DOUBLING, 0, 0, 0.0, 0}, "intervals 32/4096"},
        {8, 8, 1, {GF2E_SCHED_DOUBLING, 0, 0, 0.0, 0}, "intervals 8/8"},
        {64, 4096, 4, {GF2E_SCHED_LINEAR, 3, 0, 0.0, 0}, "block m=4 q0=3"},
        {64, 4096, 6, {GF2E_SCHED_OPT, 0, 60, 1.25, 0}, "block m=6 sched-opt G=60"}};
    for (const Pol &p : pol) {
        u64 nf = 0, nu = 0, nb = 0;
        if (run(r, surv, k0, maxd, p.L0, p.Lmax, 64, p.block, p.sched, nullptr, 0, nullptr, &nf,
                &nu, &nb))
            return 1;
        bool ok = surv.size() == 104 && nf == 102 && nu == 2 && nb == 0;
        printf("scan r=4423 k0=5 maxd=200 %s: %zu survivors, "
               "%" PRIu64 " found, %" PRIu64 " u, %" PRIu64 " not dividing  %s\n",
               p.name, surv.size(), nf, nu, nb, ok ? "PASS" : "FAIL");
        bad += !ok;
    }
    printf(bad ? "\nSCAN SELFTEST: %d FAILURES\n" : "\nSCAN SELFTEST: ALL PASS\n", bad);
    return bad ? 1 : 0;
}

int main(int argc, char **argv) {
    if (argc >= 2 && !strcmp(argv[1], "--selftest")) return selftest();
    if (argc < 6) {
        fprintf(stderr, "usage: %s <r> <survivors.txt> <k0> <maxd> <out_prefix>\n"
                        "          [--interval Lmax] [--l0 L0] [--batch B] [--block m] [--verbose 0..3]\n"
                        "          [--sched doubling|linear|opt] [--q0 N] [--sched-G N] [--sched-rho R] [--Zq N]\n"
                        "       %s --selftest\n"
                        "k0 must be the depth the coarse sieve actually reached.\n",
                argv[0], argv[0]);
        return 1;
    }
    u64 r = strtoull(argv[1], 0, 10), k0 = strtoull(argv[3], 0, 10), maxd = strtoull(argv[4], 0, 10);
    std::string prefix = argv[5];
    u64 L0 = 64, Lmax = 4096;
    int batch = 64, verbose = 1, block = 1;
    const char *state_path = nullptr;
    gf2e_sched sched{GF2E_SCHED_DOUBLING, 0, 4000, 1.25, 0};
    for (int i = 6; i < argc; i++) {
        if (!strcmp(argv[i], "--sched") && i + 1 < argc) {
            const char *v = argv[++i];
            if (!strcmp(v, "opt")) sched.mode = GF2E_SCHED_OPT;
            else if (!strcmp(v, "linear")) sched.mode = GF2E_SCHED_LINEAR;
            else if (!strcmp(v, "doubling")) sched.mode = GF2E_SCHED_DOUBLING;
            else { fprintf(stderr, "bad --sched %s (doubling|linear|opt)\n", v); return 1; }
            continue;
        }
        if (!strcmp(argv[i], "--q0") && i + 1 < argc) {
            sched.q0 = strtoull(argv[++i], 0, 10);
            if (sched.mode == GF2E_SCHED_DOUBLING) sched.mode = GF2E_SCHED_LINEAR;
            continue;
        }
        if (!strcmp(argv[i], "--sched-G") && i + 1 < argc) { sched.G = strtoull(argv[++i], 0, 10); continue; }
        if (!strcmp(argv[i], "--sched-rho") && i + 1 < argc) { sched.rho = atof(argv[++i]); continue; }
        if (!strcmp(argv[i], "--Zq") && i + 1 < argc) { sched.qcap = strtoull(argv[++i], 0, 10); continue; }
        if (!strcmp(argv[i], "--interval") && i + 1 < argc) Lmax = strtoull(argv[++i], 0, 10);
        else if (!strcmp(argv[i], "--l0") && i + 1 < argc) L0 = strtoull(argv[++i], 0, 10);
        else if (!strcmp(argv[i], "--batch") && i + 1 < argc) batch = atoi(argv[++i]);
        else if (!strcmp(argv[i], "--block") && i + 1 < argc) block = atoi(argv[++i]);
        else if (!strcmp(argv[i], "--verbose") && i + 1 < argc) verbose = atoi(argv[++i]);
        else if (!strcmp(argv[i], "--state") && i + 1 < argc) state_path = argv[++i];
        else if (!strcmp(argv[i], "--gcd-threads") && i + 1 < argc) {
            fprintf(stderr, "note: %s ignored (gcds run on the GPU)\n", argv[i]);
            i++;
        } else {
            fprintf(stderr, "unknown option %s\n", argv[i]);
            return 1;
        }
    }
    if (Lmax < 1) Lmax = 1;
    if (L0 > Lmax) L0 = Lmax;
    // tsfactor's default first interval: ceil(600 / m) blocks
    if (sched.mode != GF2E_SCHED_DOUBLING && sched.q0 == 0)
        sched.q0 = (600 + (u64)block - 1) / (u64)block;
    if (!(k0 >= 1 && maxd > k0)) { fprintf(stderr, "need 1 <= k0 < maxd\n"); return 1; }
    std::vector<u64> surv;
    FILE *f = fopen(argv[2], "r");
    if (!f) { perror(argv[2]); return 1; }
    u64 s;
    while (fscanf(f, "%" SCNu64, &s) == 1) {
        if (s >= 1 && 2 * s < r) surv.push_back(s);
        else fprintf(stderr, "skipping s=%" PRIu64 " (need 1 <= s <= (r-1)/2)\n", s);
    }
    fclose(f);
    std::string rpath = prefix + ".results.txt";
    std::set<u64> done;
    if ((f = fopen(rpath.c_str(), "r"))) {
        char line[256];
        while (fgets(line, sizeof line, f))
            if (sscanf(line, "%" SCNu64, &s) == 1) done.insert(s);
        fclose(f);
    }
    std::vector<u64> todo;
    for (u64 v : surv)
        if (!done.count(v)) todo.push_back(v);
    fprintf(stderr, "trinomial_scan r=%" PRIu64 " k0=%" PRIu64 " maxd=%" PRIu64 ": %zu survivors "
                    "(%zu already done), gcd backend: GPU, batch %d\n",
            r, k0, maxd, surv.size(), done.size(), batch);
    FILE *fres = fopen(rpath.c_str(), "a");
    if (!fres) { perror(rpath.c_str()); return 1; }
    double t0 = now_s();
    u64 nf = 0, nu = 0, nb = 0;
    int rc = todo.empty() ? 0
                          : run(r, todo, k0, maxd, L0, Lmax, batch, block, sched, fres, verbose,
                                state_path, &nf, &nu, &nb);
    fclose(fres);
    fprintf(stderr, "done: %" PRIu64 " found, %" PRIu64 " u, %.1fs total%s\n", nf, nu,
            now_s() - t0, nb ? " (WARNING: some factors failed verification)" : "");
    return rc ? rc : (nb ? 1 : 0);
}
