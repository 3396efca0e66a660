// bin2cert -- a found.bin image (coarse_sieve --found) back to certificate
// text (the reference's bin2cert.c): line s is "s u" for an all-ones record,
// else "s d p<hex>" with d the top 16 bits and the mask the low 48.
//
//   bin2cert <binary_file> > out.found.cert
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "certfmt.h"

typedef uint64_t u64;

int main(int argc, char **argv) {
    if (argc != 2) {
        fprintf(stderr, "Usage: %s <binary_file>\n", argv[0]);
        return 1;
    }
    FILE *f = fopen(argv[1], "rb");
    if (!f) { perror("Error opening file"); return 1; }
    // records in rounds of 2^22, each round's lines formatted by several
    // threads (certfmt.h) and written in order
    std::vector<u64> rec((size_t)1 << 22);
    u64 s = 1;
    for (size_t n; (n = fread(rec.data(), 8, rec.size(), f)) > 0; s += n)
        if (certfmt::write_lines(stdout, rec.data(), n, s, certfmt::Lines::Bin2Cert) < 0) {
            fclose(f);
            return 1;
        }
    const bool bad = ferror(f);
    fclose(f);
    if (bad) { fprintf(stderr, "Error reading from file.\n"); return 1; }
    return 0;
}
