// polyhost.h -- host-side GF(2)[x] arithmetic for resolving a hit: the
// interval gcd g of a deep scan is factored far enough to give its least
// irreducible factor (trinomial_scan.cu:283-325 via gf2_gcd_ntl.cpp:68-92,
// tsfactor.cu:928-974).  Plain C++ (no CUDA); word arrays, least
// significant word first, bit i of word w is the coefficient of x^(64 w + i).
#pragma once

#include <cstdint>
#include <vector>

namespace gf2e {
namespace hostpoly {

typedef std::vector<uint64_t> Poly;

long long deg(const Poly &a);                 // -1 for the zero polynomial
void trim(Poly &a);                           // drop zero top words
Poly mul(const Poly &a, const Poly &b);       // carry-less product
Poly gcd(Poly a, Poly b);
Poly divide(const Poly &a, const Poly &b);    // exact quotient a / b

// Arithmetic modulo a fixed g of degree n >= 1 (Barrett reduction with
// mu = floor(x^(2n) / g); exact for inputs of degree < 2n).
class Modulus {
public:
    explicit Modulus(const Poly &g);
    long long degree() const { return n_; }
    const Poly &poly() const { return g_; }
    Poly reduce(const Poly &p) const;                 // p mod g, any degree
    Poly sqr(const Poly &a) const;                    // a^2 mod g, a reduced
    Poly mul(const Poly &a, const Poly &b) const;     // a b mod g, both reduced
private:
    Poly reduce2n(Poly p) const;                      // deg p < 2n
    Poly g_, mu_;
    long long n_;
};

// Least irreducible factor of g (squarefree, as every divisor of a
// trinomial is): the least k <= kmax with gcd(x^(2^k) + x, g) != 1 and the
// numerically least irreducible factor of degree k.  The caller may state
// that g has no factor of degree <= clean_below; k <= clean_below is then
// not tested, and when deg g < 2 (clean_below + 1) g is itself irreducible
// (two factors would need degree >= 2 (clean_below + 1)).  false when no
// factor has degree <= kmax.
bool least_factor(const Poly &g, uint64_t clean_below, uint64_t kmax, uint64_t &d_out,
                  Poly &mask);

}  // namespace hostpoly
}  // namespace gf2e
