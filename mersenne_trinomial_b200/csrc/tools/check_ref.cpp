// check_ref -- cross-check sieve output against reference factor lists
// (the reference's check_ref.cpp, same options and verdicts):
//
//   check_ref --ref <reference.txt> [--smax S] [--dmin D] [--dmax D]
//             [--cert <f.found.cert>]... [--survivors <f.survivors.txt>]
//             [--found <f.found.bin>]
//
// The reference lists "s d p<hex>" for degrees in [dmin, dmax] (default
// 30..34).  The sieve's view of each s is assembled from the survivors file
// (no factor), the certificates (least key wins) and a found.bin image.
// Reported: false negatives (reference factor, sieve survivor), degree and
// polynomial mismatches, s the sieve resolves below the reference's range,
// reference s with no sieve data, and in-range sieve factors the reference
// lacks.  Exit 1 and "*** DISCREPANCIES FOUND ***" if any check fails, else
// "ALL CHECKS PASSED".
//
// Input lines are read as fgets(buf, 512) would return them and parsed by
// several threads (lines.h); each line is read either by a fast path for
// the canonical forms ("s d p<hex>", "s"), whose result equals that of the
// sscanf / strtoull calls below, or by those calls themselves, and the
// lines are applied in file order.  At r = 136279841 that is 64 M
// certificate lines in seconds instead of a quarter of a minute.
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>

#include "lines.h"

typedef uint64_t u64;

namespace {
constexpr u64 SURVIVOR = ~0ull;   // no factor
constexpr u64 NO_DATA = 0;        // nothing supplied for this s

// "s d p<hex>" -> (s, d, mask); false for other lines
bool parse_factor(const char *line, u64 &s, int &d, u64 &mask) {
    char hex[128];
    unsigned long long ss;
    if (sscanf(line, "%llu %d p%127s", &ss, &d, hex) != 3) return false;
    s = ss;
    mask = strtoull(hex, nullptr, 16);
    return true;
}

bool dig(char c) { return c >= '0' && c <= '9'; }
int hexd(char c) { return dig(c) ? c - '0' : (c >= 'a' && c <= 'f') ? c - 'a' + 10 : -1; }

// One fgets chunk of a certificate or reference file.  The fast path takes
// exactly "S D pH" with an optional final newline, S of 1..19 digits, D of
// 1..9, H of 1..16 lowercase hex digits: no value can overflow there, so it
// gives what parse_factor gives.  Anything else goes to parse_factor.
struct Factor {
    u64 s, mask;
    int d;
};
bool factor_chunk(const char *p, size_t n, Factor &f) {
    size_t i = 0, j;
    u64 s = 0, mask = 0;
    int d = 0;
    for (j = i; j < n && j - i < 20 && dig(p[j]); j++) s = s * 10 + (u64)(p[j] - '0');
    bool fast = j > i && j - i <= 19 && j < n && p[j] == ' ';
    if (fast) {
        i = j + 1;
        for (j = i; j < n && j - i < 10 && dig(p[j]); j++) d = d * 10 + (p[j] - '0');
        fast = j > i && j - i <= 9 && j + 1 < n && p[j] == ' ' && p[j + 1] == 'p';
    }
    if (fast) {
        i = j + 2;
        int h = 0;
        for (j = i; j < n && j - i < 17 && (h = hexd(p[j])) >= 0; j++) mask = (mask << 4) | (u64)h;
        fast = j > i && j - i <= 16 && (j == n || (j + 1 == n && p[j] == '\n'));
    }
    if (fast) {
        f.s = s;
        f.d = d;
        f.mask = mask;
        return true;
    }
    char line[lines::kFgetsBytes + 1];
    lines::c_string(p, n, line);
    return parse_factor(line, f.s, f.d, f.mask);
}

// One fgets chunk of a survivors file: strtoull(line, &end, 10), fast for
// 1..19 digits and an optional newline.  Every chunk yields a record; `ok`
// is end != line.
struct Surv {
    u64 s;
    bool ok;
};
bool surv_chunk(const char *p, size_t n, Surv &r) {
    size_t j = 0;
    u64 s = 0;
    for (; j < n && j < 20 && dig(p[j]); j++) s = s * 10 + (u64)(p[j] - '0');
    if (j > 0 && j <= 19 && (j == n || (j + 1 == n && p[j] == '\n'))) {
        r.s = s;
        r.ok = true;
        return true;
    }
    char line[lines::kFgetsBytes + 1];
    lines::c_string(p, n, line);
    char *end = nullptr;
    r.s = strtoull(line, &end, 10);
    r.ok = end != line;
    return true;
}
}  // namespace

int main(int argc, char **argv) {
    const char *ref_path = nullptr, *surv_path = nullptr, *found_path = nullptr;
    std::vector<const char *> certs;
    u64 smax = 0;
    int dmin = 30, dmax = 34;
    for (int a = 1; a < argc; a++) {
        const bool val = a + 1 < argc;
        if (!strcmp(argv[a], "--ref") && val) ref_path = argv[++a];
        else if (!strcmp(argv[a], "--cert") && val) certs.push_back(argv[++a]);
        else if (!strcmp(argv[a], "--survivors") && val) surv_path = argv[++a];
        else if (!strcmp(argv[a], "--found") && val) found_path = argv[++a];
        else if (!strcmp(argv[a], "--smax") && val) smax = strtoull(argv[++a], nullptr, 10);
        else if (!strcmp(argv[a], "--dmin") && val) dmin = atoi(argv[++a]);
        else if (!strcmp(argv[a], "--dmax") && val) dmax = atoi(argv[++a]);
        else { fprintf(stderr, "unknown argument '%s'\n", argv[a]); return 1; }
    }
    if (!ref_path || (certs.empty() && !found_path)) {
        fprintf(stderr,
                "usage: %s --ref <reference.txt> [--smax S] [--dmin D] [--dmax D]\n"
                "          [--cert <f.found.cert>]... [--survivors <f.survivors.txt>]\n"
                "          [--found <f.found.bin>]\n", argv[0]);
        return 1;
    }
    const int threads = lines::default_threads();
    // reference lines in the degree range (they also fix smax if not given)
    std::map<u64, std::pair<int, u64>> ref;
    u64 ref_lines = 0, ref_top = 0;
    {
        FILE *f = fopen(ref_path, "r");
        if (!f) { perror(ref_path); return 1; }
        lines::for_each<Factor>(f, factor_chunk, [&](const Factor &x) {
            if (x.d < dmin || x.d > dmax) return;
            ref[x.s] = {x.d, x.mask};
            ref_lines++;
            if (x.s > ref_top) ref_top = x.s;
        }, threads);
        fclose(f);
    }
    if (!smax) smax = ref_top;
    std::vector<u64> view(smax + 1, NO_DATA);
    u64 n_surv = 0, n_cert = 0;
    if (surv_path) {
        FILE *f = fopen(surv_path, "r");
        if (!f) { perror(surv_path); return 1; }
        lines::for_each<Surv>(f, surv_chunk, [&](const Surv &x) {
            if (!x.ok || x.s < 1 || x.s > smax) return;
            view[x.s] = SURVIVOR;
            n_surv++;
        }, threads);
        fclose(f);
    }
    for (const char *path : certs) {
        FILE *f = fopen(path, "r");
        if (!f) { perror(path); return 1; }
        lines::for_each<Factor>(f, factor_chunk, [&](const Factor &x) {
            if (x.s < 1 || x.s > smax) return;
            const u64 key = ((u64)x.d << 48) | x.mask;
            if (view[x.s] == SURVIVOR)
                printf("INCONSISTENT INPUT: s=%" PRIu64 " is in %s but also in the survivors file\n",
                       x.s, path);
            if (view[x.s] == NO_DATA || key < view[x.s]) view[x.s] = key;
            n_cert++;
        }, threads);
        fclose(f);
    }
    if (found_path) {
        FILE *f = fopen(found_path, "rb");
        if (!f) { perror(found_path); return 1; }
        std::vector<u64> img(smax);
        if (fread(img.data(), 8, smax, f) != smax) {
            fprintf(stderr, "%s: short read (is --smax right?)\n", found_path);
            return 1;
        }
        fclose(f);
        for (u64 s = 1; s <= smax; s++) {
            const u64 v = img[s - 1];
            if (v == SURVIVOR) { if (view[s] == NO_DATA) view[s] = SURVIVOR; }
            else if (v != NO_DATA && (view[s] == NO_DATA || v < view[s])) view[s] = v;
        }
    }
    u64 false_neg = 0, deg_bad = 0, poly_bad = 0, below = 0, agree = 0, no_data = 0;
    for (const auto &kv : ref) {
        const u64 s = kv.first;
        const int d = kv.second.first;
        const u64 mask = kv.second.second;
        if (s > smax) continue;
        const u64 v = view[s];
        if (v == SURVIVOR) {
            if (++false_neg <= 10)
                printf("FALSE NEGATIVE: s=%" PRIu64 " is a survivor but reference has degree %d\n", s, d);
            continue;
        }
        if (v == NO_DATA) { no_data++; continue; }
        const int vd = (int)(v >> 48);
        const u64 vm = v & 0xFFFFFFFFFFFFull;
        if (vd < d) { below++; continue; }
        if (vd != d) {
            if (++deg_bad <= 10) printf("DEGREE MISMATCH: s=%" PRIu64 " sieve=%d reference=%d\n", s, vd, d);
            continue;
        }
        if (vm != mask) {
            if (++poly_bad <= 10)
                printf("POLYNOMIAL MISMATCH: s=%" PRIu64 " d=%d sieve=0x%" PRIx64 " ref=0x%" PRIx64 "\n",
                       s, d, vm, mask);
            continue;
        }
        agree++;
    }
    u64 false_pos = 0;
    const u64 hi = ref_top < smax ? ref_top : smax;
    for (u64 s = 1; s <= hi; s++) {
        const u64 v = view[s];
        if (v == SURVIVOR || v == NO_DATA) continue;
        const int vd = (int)(v >> 48);
        if (vd < dmin || vd > dmax || ref.count(s)) continue;
        if (++false_pos <= 10)
            printf("NOT IN REFERENCE: s=%" PRIu64 " sieve reports degree %d\n", s, vd);
    }
    printf("\nreference lines in [%d,%d]: %" PRIu64 "  (s up to %" PRIu64 ")\n", dmin, dmax,
           ref_lines, ref_top);
    printf("sieve input: %" PRIu64 " cert lines, %" PRIu64 " survivors; checked s = 1..%" PRIu64 "\n",
           n_cert, n_surv, hi);
    printf("  exact agreement (degree + polynomial): %" PRIu64 "\n", agree);
    printf("  sieve found a SMALLER degree (below ref range): %" PRIu64 "\n", below);
    printf("  reference s with no data supplied (add more certs): %" PRIu64 "\n", no_data);
    printf("  FALSE NEGATIVES (ref has factor, sieve says survivor): %" PRIu64 "\n", false_neg);
    printf("  degree mismatches: %" PRIu64 "\n", deg_bad);
    printf("  polynomial mismatches: %" PRIu64 "\n", poly_bad);
    printf("  sieve in-range but absent from reference: %" PRIu64 "\n", false_pos);
    const bool bad = false_neg || deg_bad || poly_bad || false_pos;
    printf("\n%s\n", bad ? "*** DISCREPANCIES FOUND ***" : "ALL CHECKS PASSED");
    return bad ? 1 : 0;
}
