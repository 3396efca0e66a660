// polyhost.cpp -- host GF(2)[x] arithmetic for hit resolution.
//
// Products use the x86 carry-less multiply (PCLMULQDQ) on 64-bit words,
// Karatsuba above a small schoolbook size; the portable loop is taken when
// the CPU lacks the instruction.  Reduction modulo a fixed g is Barrett's
// (mu = floor(x^(2n)/g), two products per reduction), so x^(2^k) mod g
// costs a squaring and two products of n-bit operands instead of the n
// shift-XORs of long division.  The least-degree search accumulates
// (x^(2^k) + x) over blocks of k and takes one gcd per block, walking back
// through the block only when that gcd is non-trivial (the reference's
// fallback and NTL's DDF test every k, gf2_gcd_ntl.cpp:68-92).
#include "polyhost.h"

#include <immintrin.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>

namespace gf2e {
namespace hostpoly {
namespace {

typedef uint64_t u64;

__attribute__((target("pclmul,sse4.1"))) inline void clmul_hw(u64 a, u64 b, u64 &lo,
                                                               u64 &hi) {
    const __m128i r = _mm_clmulepi64_si128(_mm_cvtsi64_si128((long long)a),
                                           _mm_cvtsi64_si128((long long)b), 0);
    lo = (u64)_mm_cvtsi128_si64(r);
    hi = (u64)_mm_extract_epi64(r, 1);
}

inline void clmul_sw(u64 a, u64 b, u64 &lo, u64 &hi) {
    u64 l = 0, h = 0;
    for (int i = 0; i < 64; i++)
        if ((b >> i) & 1) {
            l ^= a << i;
            if (i) h ^= a >> (64 - i);
        }
    lo = l;
    hi = h;
}

// GF2E_NO_PCLMUL=1 forces the portable loop (used to test it)
bool have_pclmul() {
    static const bool ok = __builtin_cpu_supports("pclmul") && __builtin_cpu_supports("sse4.1") &&
                           !(std::getenv("GF2E_NO_PCLMUL") && std::getenv("GF2E_NO_PCLMUL")[0] == '1');
    return ok;
}

// c[0 .. na+nb) ^= a[0 .. na) * b[0 .. nb), schoolbook
__attribute__((target("pclmul,sse4.1"))) void school_hw(const u64 *a, size_t na, const u64 *b,
                                                        size_t nb, u64 *c) {
    for (size_t i = 0; i < na; i++) {
        const u64 ai = a[i];
        if (!ai) continue;
        for (size_t j = 0; j < nb; j++) {
            u64 lo, hi;
            clmul_hw(ai, b[j], lo, hi);
            c[i + j] ^= lo;
            c[i + j + 1] ^= hi;
        }
    }
}

void school_sw(const u64 *a, size_t na, const u64 *b, size_t nb, u64 *c) {
    for (size_t i = 0; i < na; i++) {
        if (!a[i]) continue;
        for (size_t j = 0; j < nb; j++) {
            u64 lo, hi;
            clmul_sw(a[i], b[j], lo, hi);
            c[i + j] ^= lo;
            c[i + j + 1] ^= hi;
        }
    }
}

constexpr size_t KARA_MIN = 24;       // words: schoolbook below

// c[0 .. 2n) ^= a * b, both n words; scratch of 4n words
void kara(const u64 *a, const u64 *b, size_t n, u64 *c, u64 *scratch, bool hw) {
    if (n < KARA_MIN) {
        if (hw) school_hw(a, n, b, n, c);
        else school_sw(a, n, b, n, c);
        return;
    }
    const size_t h = n / 2, hh = n - h;          // low h words, high hh >= h words
    // t = (a0 + a1)(b0 + b1), p0 = a0 b0, p2 = a1 b1
    u64 *sa = scratch, *sb = scratch + hh, *t = scratch + 2 * hh;
    u64 *rest = t + 2 * hh;
    for (size_t i = 0; i < hh; i++) {
        sa[i] = a[h + i] ^ (i < h ? a[i] : 0);
        sb[i] = b[h + i] ^ (i < h ? b[i] : 0);
    }
    std::memset(t, 0, 2 * hh * sizeof(u64));
    kara(sa, sb, hh, t, rest, hw);
    // p0 into a zeroed temporary region, p2 likewise, reusing sa/sb space
    std::vector<u64> p0(2 * h, 0), p2(2 * hh, 0);
    kara(a, b, h, p0.data(), rest, hw);
    kara(a + h, b + h, hh, p2.data(), rest, hw);
    for (size_t i = 0; i < 2 * h; i++) {
        c[i] ^= p0[i];
        t[i] ^= p0[i];
    }
    for (size_t i = 0; i < 2 * hh; i++) {
        c[2 * h + i] ^= p2[i];
        t[i] ^= p2[i];
    }
    for (size_t i = 0; i < 2 * hh; i++) c[h + i] ^= t[i];
}

// a ^= b << sh (a grown as needed)
void xor_shift(Poly &a, const Poly &b, u64 sh) {
    const size_t ws = (size_t)(sh >> 6);
    const unsigned bs = (unsigned)(sh & 63);
    if (a.size() < b.size() + ws + 1) a.resize(b.size() + ws + 1, 0);
    for (size_t j = 0; j < b.size(); j++) {
        a[j + ws] ^= b[j] << bs;
        if (bs) a[j + ws + 1] ^= b[j] >> (64 - bs);
    }
}

// floor(a / x^k)
Poly shr(const Poly &a, u64 k) {
    const size_t ws = (size_t)(k >> 6);
    const unsigned bs = (unsigned)(k & 63);
    if (ws >= a.size()) return Poly();
    Poly o(a.size() - ws, 0);
    for (size_t i = 0; i < o.size(); i++) {
        u64 v = a[i + ws] >> bs;
        if (bs && i + ws + 1 < a.size()) v |= a[i + ws + 1] << (64 - bs);
        o[i] = v;
    }
    trim(o);
    return o;
}

// a mod x^k
void truncate(Poly &a, u64 k) {
    const size_t nw = (size_t)((k + 63) >> 6);
    if (a.size() > nw) a.resize(nw);
    if ((k & 63) && a.size() == nw) a[nw - 1] &= (1ull << (k & 63)) - 1;
    trim(a);
}

// degree of a at or below bit `from` (a has no set bit above it)
long long deg_below(const Poly &a, long long from) {
    for (long long i = from >> 6; i >= 0; i--)
        if (a[(size_t)i]) return i * 64 + 63 - __builtin_clzll(a[(size_t)i]);
    return -1;
}

// a mod b by long division: one shift-XOR of b's words per quotient bit,
// the degree of a tracked downwards instead of rescanned
void mod_slow(Poly &a, const Poly &b_in) {
    Poly b = b_in;
    trim(b);
    const long long db = deg(b);
    long long da = deg(a);
    const size_t bw = b.size();
    if (da >= 0 && a.size() < (size_t)(da >> 6) + 2) a.resize((size_t)(da >> 6) + 2, 0);
    while (da >= db) {
        const u64 sh = (u64)(da - db);
        const size_t ws = (size_t)(sh >> 6);
        const unsigned bs = (unsigned)(sh & 63);
        if (bs) {
            // the spill word past a's top is zero (one padding word)
            for (size_t j = 0; j < bw; j++) {
                a[j + ws] ^= b[j] << bs;
                a[j + ws + 1] ^= b[j] >> (64 - bs);
            }
        } else {
            for (size_t j = 0; j < bw; j++) a[j + ws] ^= b[j];
        }
        da = deg_below(a, da);
    }
    trim(a);
}

Poly spread_sqr(const Poly &a) {
    Poly c(2 * a.size(), 0);
    for (size_t i = 0; i < a.size(); i++)
        for (int h = 0; h < 2; h++) {
            u64 x = (a[i] >> (32 * h)) & 0xFFFFFFFFull;
            x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
            x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
            x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
            x = (x | (x << 2)) & 0x3333333333333333ull;
            x = (x | (x << 1)) & 0x5555555555555555ull;
            c[2 * i + h] = x;
        }
    trim(c);
    return c;
}

bool less_than(const Poly &x, const Poly &y) {
    const size_t n = std::max(x.size(), y.size());
    for (size_t i = n; i-- > 0;) {
        const u64 xv = i < x.size() ? x[i] : 0, yv = i < y.size() ? y[i] : 0;
        if (xv != yv) return xv < yv;
    }
    return false;
}

u64 rng_next(u64 &st) {
    u64 z = (st += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// split g (a product of distinct irreducibles of degree d) into its
// factors with the trace map: for random u, Tr(u) = u + u^2 + ... +
// u^(2^(d-1)) mod g is 0 or 1 modulo each factor, so gcd(Tr(u), g) splits g
// about half the time (Cantor-Zassenhaus for characteristic 2)
void edf_split(const Poly &g, u64 d, u64 &rng, std::vector<Poly> &out, int depth = 0) {
    const long long dg = deg(g);
    if (dg <= 0) return;
    if ((u64)dg == d || depth > 200) {
        out.push_back(g);
        return;
    }
    const Modulus M(g);
    for (int tries = 0; tries < 64; tries++) {
        Poly u((size_t)(dg / 64) + 1, 0);
        for (auto &w : u) w = rng_next(rng);
        if (dg % 64 != 63) u.back() &= (1ull << (dg % 64 + 1)) - 1;
        u = M.reduce(u);
        Poly t = u, acc = u;
        for (u64 i = 1; i < d; i++) {
            t = M.sqr(t);
            if (acc.size() < t.size()) acc.resize(t.size(), 0);
            for (size_t j = 0; j < t.size(); j++) acc[j] ^= t[j];
        }
        trim(acc);
        const Poly h = gcd(g, acc);
        const long long dh = deg(h);
        if (dh > 0 && dh < dg) {
            edf_split(h, d, rng, out, depth + 1);
            edf_split(divide(g, h), d, rng, out, depth + 1);
            return;
        }
    }
    out.push_back(g);           // not split: reported as is (caller checks degree)
}

// the numerically least irreducible factor of degree d of gk (a product of
// such factors); false if the splitting did not isolate factors of degree d
bool least_of_degree(const Poly &gk, u64 d, Poly &mask) {
    if ((u64)deg(gk) == d) {
        mask = gk;
        trim(mask);
        return true;
    }
    std::vector<Poly> parts;
    u64 rng = 0x243F6A8885A308D3ull ^ d;
    edf_split(gk, d, rng, parts);
    bool have = false;
    for (auto &p : parts) {
        if ((u64)deg(p) != d) return false;
        if (!have || less_than(p, mask)) {
            mask = p;
            have = true;
        }
    }
    trim(mask);
    return have;
}

}  // namespace

long long deg(const Poly &a) {
    for (size_t i = a.size(); i-- > 0;)
        if (a[i]) return (long long)(i * 64 + 63 - __builtin_clzll(a[i]));
    return -1;
}

void trim(Poly &a) {
    while (!a.empty() && !a.back()) a.pop_back();
}

Poly mul(const Poly &a_in, const Poly &b_in) {
    Poly a = a_in, b = b_in;
    trim(a);
    trim(b);
    if (a.empty() || b.empty()) return Poly();
    const bool hw = have_pclmul();
    Poly c(a.size() + b.size() + 1, 0);
    if (a.size() < KARA_MIN || b.size() < KARA_MIN) {
        if (hw) school_hw(a.data(), a.size(), b.data(), b.size(), c.data());
        else school_sw(a.data(), a.size(), b.data(), b.size(), c.data());
        trim(c);
        return c;
    }
    // unequal lengths: Karatsuba on equal-length slices of the longer one
    if (a.size() < b.size()) std::swap(a, b);
    const size_t n = b.size();
    std::vector<u64> scratch(8 * n + 64), part(2 * n);
    for (size_t off = 0; off < a.size(); off += n) {
        const size_t len = std::min(n, a.size() - off);
        std::fill(part.begin(), part.end(), 0);
        if (len == n) {
            kara(a.data() + off, b.data(), n, part.data(), scratch.data(), hw);
        } else if (hw) {
            school_hw(a.data() + off, len, b.data(), n, part.data());
        } else {
            school_sw(a.data() + off, len, b.data(), n, part.data());
        }
        for (size_t i = 0; i < 2 * n && off + i < c.size(); i++) c[off + i] ^= part[i];
    }
    trim(c);
    return c;
}

Poly gcd(Poly a, Poly b) {
    trim(a);
    trim(b);
    while (!b.empty()) {
        mod_slow(a, b);
        std::swap(a, b);
    }
    return a;
}

Poly divide(const Poly &a, const Poly &b) {
    const long long db = deg(b);
    Poly rem = a, quo;
    long long dr = deg(rem);
    if (db < 0 || dr < db) return Poly();
    quo.assign((size_t)((dr - db) / 64) + 1, 0);
    while (dr >= db) {
        const u64 sh = (u64)(dr - db);
        quo[sh >> 6] |= 1ull << (sh & 63);
        xor_shift(rem, b, sh);
        dr = deg(rem);
    }
    trim(quo);
    return quo;
}

Modulus::Modulus(const Poly &g) : g_(g), n_(deg(g)) {
    trim(g_);
    // mu = floor(x^(2n) / g)
    if (n_ >= 1) {
        Poly x2n((size_t)((2 * n_) / 64) + 1, 0);
        x2n[(size_t)(2 * n_) >> 6] = 1ull << ((2 * n_) & 63);
        mu_ = divide(x2n, g_);
    }
}

Poly Modulus::reduce2n(Poly p) const {
    // q = floor(floor(p / x^n) * mu / x^n); p - q g has degree < n
    trim(p);
    if (deg(p) < n_) return p;
    const Poly q = shr(hostpoly::mul(shr(p, (u64)n_), mu_), (u64)n_);
    const Poly qg = hostpoly::mul(q, g_);
    if (p.size() < qg.size()) p.resize(qg.size(), 0);
    for (size_t i = 0; i < qg.size(); i++) p[i] ^= qg[i];
    truncate(p, (u64)n_);
    return p;
}

Poly Modulus::reduce(const Poly &p_in) const {
    Poly p = p_in;
    trim(p);
    if (n_ < 1) return Poly();
    // fold the part above 2n in n-bit pieces from the top, each step a
    // reduction of a value below 2n
    while (deg(p) >= 2 * n_) {
        const long long dp = deg(p);
        const u64 cut = (u64)(dp - 2 * n_ + 1);      // low bits kept aside
        Poly lo = p;
        truncate(lo, cut);
        Poly hi = reduce2n(shr(p, cut));             // (p >> cut) mod g
        // p = hi * x^cut + lo, deg < n + cut <= dp - n + 1
        p = lo;
        xor_shift(p, hi, cut);
        trim(p);
    }
    return reduce2n(p);
}

Poly Modulus::sqr(const Poly &a) const { return reduce2n(spread_sqr(a)); }

Poly Modulus::mul(const Poly &a, const Poly &b) const { return reduce2n(hostpoly::mul(a, b)); }

bool least_factor(const Poly &g_in, uint64_t clean_below, uint64_t kmax, uint64_t &d_out,
                  Poly &mask) {
    Poly g = g_in;
    trim(g);
    const long long n = deg(g);
    if (n <= 0) return false;
    if (clean_below > 0 && (u64)n < 2 * (clean_below + 1)) {
        // every factor has degree > clean_below, so two would exceed deg g
        d_out = (u64)n;
        mask = g;
        return true;
    }
    const Modulus M(g);
    const Poly x{2};
    Poly h = M.reduce(x);                        // x^(2^k) mod g, k = 0
    constexpr u64 BLOCK = 32;
    std::vector<Poly> block;                     // x^(2^k) + x mod g of the block
    block.reserve(BLOCK);
    Poly acc{1};
    u64 k0 = 0;
    for (u64 k = 1; k <= kmax; k++) {
        h = M.sqr(h);
        if (k <= clean_below) continue;
        Poly hx = h;
        if (hx.empty()) hx.push_back(0);
        hx[0] ^= 2;
        trim(hx);
        if (block.empty()) k0 = k;
        acc = M.mul(acc, hx);
        block.push_back(hx);
        if (block.size() < BLOCK && k < kmax) continue;
        if (deg(gcd(g, acc)) > 0) {
            for (size_t i = 0; i < block.size(); i++) {
                const Poly gk = gcd(g, block[i]);
                if (deg(gk) > 0) {
                    d_out = k0 + i;
                    return least_of_degree(gk, d_out, mask);
                }
            }
            return false;               // the product saw a factor no single k did
        }
        block.clear();
        acc.assign(1, 1);
    }
    return false;
}

}  // namespace hostpoly
}  // namespace gf2e
