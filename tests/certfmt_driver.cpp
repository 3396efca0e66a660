// Test driver for the result formatter (mersenne_trinomial_b200/csrc/tools/
// certfmt.h), compiled by tests/test_certfmt.py.  Host only.
//
//   certfmt_driver <cert|survivors|bin2cert> <keys.bin> <s_of_first> <threads>
//
// keys.bin holds LE u64 keys; the lines go to stdout, the line count to stderr.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "certfmt.h"

int main(int argc, char **argv) {
    if (argc != 5) return 2;
    certfmt::Lines kind;
    if (!strcmp(argv[1], "cert")) kind = certfmt::Lines::Cert;
    else if (!strcmp(argv[1], "survivors")) kind = certfmt::Lines::Survivors;
    else if (!strcmp(argv[1], "bin2cert")) kind = certfmt::Lines::Bin2Cert;
    else return 2;
    FILE *f = fopen(argv[2], "rb");
    if (!f) return 2;
    std::vector<certfmt::u64> keys;
    certfmt::u64 v;
    while (fread(&v, 8, 1, f) == 1) keys.push_back(v);
    fclose(f);
    const long long n = certfmt::write_lines(stdout, keys.data(), keys.size(),
                                             strtoull(argv[3], 0, 10), kind, atoi(argv[4]));
    fprintf(stderr, "%lld\n", n);
    return n < 0 ? 1 : 0;
}
