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
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>

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
    char line[512];
    // reference lines in the degree range (they also fix smax if not given)
    std::map<u64, std::pair<int, u64>> ref;
    u64 ref_lines = 0, ref_top = 0;
    {
        FILE *f = fopen(ref_path, "r");
        if (!f) { perror(ref_path); return 1; }
        while (fgets(line, sizeof line, f)) {
            u64 s, mask;
            int d;
            if (!parse_factor(line, s, d, mask) || d < dmin || d > dmax) continue;
            ref[s] = {d, mask};
            ref_lines++;
            if (s > ref_top) ref_top = s;
        }
        fclose(f);
    }
    if (!smax) smax = ref_top;
    std::vector<u64> view(smax + 1, NO_DATA);
    u64 n_surv = 0, n_cert = 0;
    if (surv_path) {
        FILE *f = fopen(surv_path, "r");
        if (!f) { perror(surv_path); return 1; }
        while (fgets(line, sizeof line, f)) {
            char *end = nullptr;
            const u64 s = strtoull(line, &end, 10);
            if (end == line || s < 1 || s > smax) continue;
            view[s] = SURVIVOR;
            n_surv++;
        }
        fclose(f);
    }
    for (const char *path : certs) {
        FILE *f = fopen(path, "r");
        if (!f) { perror(path); return 1; }
        while (fgets(line, sizeof line, f)) {
            u64 s, mask;
            int d;
            if (!parse_factor(line, s, d, mask) || s < 1 || s > smax) continue;
            const u64 key = ((u64)d << 48) | mask;
            if (view[s] == SURVIVOR)
                printf("INCONSISTENT INPUT: s=%" PRIu64 " is in %s but also in the survivors file\n",
                       s, path);
            if (view[s] == NO_DATA || key < view[s]) view[s] = key;
            n_cert++;
        }
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
