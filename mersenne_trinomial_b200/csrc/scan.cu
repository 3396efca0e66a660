// scan.cu -- the host-side resolution of a deep-scan hit behind the C ABI
// (trinomial_scan.cu:283-325, gf2_gcd_ntl.cpp:68-92, tsfactor.cu:928-974).
//
// A non-trivial interval gcd g = gcd(ACC, T) holds exactly the irreducible
// factors of T whose degree divides some k of the interval; the least k with
// gcd(x^(2^k) + x, g) != 1 is the least factor degree, and equal-degree
// splitting of that gcd gives the numerically least factor of that degree.
// The arithmetic is in polyhost.cpp; the scanner (scanner.cu) calls it with
// the degrees its clear intervals already exclude.
#include "gf2e_internal.cuh"
#include "polyhost.h"

#include <vector>

namespace gf2e {

// least k in [1, kmax] with gcd(x^(2^k) + x, g) != 1, and the numerically
// least irreducible factor of that degree; false if none.  Every k from 1 is
// checked, so the answer is the least factor degree of g even when g also
// holds factors below kmin (input that was not a genuine survivor, which the
// reference reports with a warning, trinomial_scan.cu:288-296).
bool resolve_factor(const std::vector<u64> &g, u64 kmin, u64 kmax, u64 &d_out,
                    std::vector<u64> &mask) {
    (void)kmin;
    return hostpoly::least_factor(g, 0, kmax, d_out, mask);
}

}  // namespace gf2e

extern "C" {

int gf2e_resolve_factor(const uint64_t *g_host, size_t gw, uint64_t kmin, uint64_t kmax,
                        uint64_t *d_out, uint64_t *mask_host, size_t mask_cap_words,
                        size_t *mask_words) {
    if (!g_host || !d_out || !mask_host || !mask_words) return gf2e::invalid("null argument");
    std::vector<u64> g(g_host, g_host + gw), mask;
    u64 d = 0;
    if (!gf2e::resolve_factor(g, kmin, kmax, d, mask)) {
        *d_out = 0;
        *mask_words = 0;
        return gf2e::invalid("no factor with degree in [%llu, %llu]",
                             (unsigned long long)kmin, (unsigned long long)kmax);
    }
    if (mask.size() > mask_cap_words) return gf2e::invalid("mask needs %zu words", mask.size());
    *d_out = d;
    for (size_t i = 0; i < mask_cap_words; i++) mask_host[i] = i < mask.size() ? mask[i] : 0;
    *mask_words = mask.size();
    return GF2E_OK;
}

}  // extern "C"
