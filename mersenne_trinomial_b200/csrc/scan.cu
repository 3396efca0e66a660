// scan.cu -- the deep scan of sieve survivors (trinomial_scan.cu:240-381)
// batched over many s on one GPU, and the host-side resolution of a hit
// (trinomial_scan.cu:208-235, gf2_gcd_ntl.cpp:68-92, tsfactor.cu:932-974).
//
// Per s: F_k = x^(2^k) mod T, T = x^r + x^s + 1, ramped to k0; then for each
// degree k the running product ACC *= (F_k + x) mod T; at the end of every
// interval (lengths L0, 2 L0, ... capped at Lmax, as the reference) one gcd
// g = gcd(ACC, T).  A non-trivial g holds exactly the irreducible factors of
// T whose degree lies in the interval (earlier intervals were clear), so the
// first hit gives the least degree: the first k in the interval with
// gcd(x^(2^k) + x, g) != 1, and the numerically least factor of that degree
// by equal-degree splitting of that gcd.
//
// B200 mapping: up to `batch` s values are resident at once (F, ACC, FFT
// buffers on the device).  Every degree step is one batched squaring launch,
// one batched transform per operand pass (blockIdx.y = state), one pointwise
// multiply, one batched overlap-add and one batched fold, for all resident
// s.  Interval-end gcds run as one batched gcd launch (one CTA per s).  When
// an s retires its slot is refilled from the queue (its own k and interval
// schedule), and when the queue is empty the slots are compacted so no work
// is spent on retired states.
#include "gf2e_internal.cuh"

#include <algorithm>
#include <cstring>
#include <vector>

namespace gf2e {
int trin_square_states(const u64 *in, u64 *out, size_t stride, int nstates, u64 r,
                       const u64 *s_dev, cudaStream_t st);
int trin_set_const(u64 *states, size_t stride, int nstates, u64 r, u64 w0, cudaStream_t st);
int trin_reduce_batch(const u64 *P, size_t pstride, size_t pw, u64 L, u64 *out, size_t ostride,
                      u64 r, const u64 *s_dev, int batch, cudaStream_t st);
int fft_fwd_packed_batch(const gf2e_fft_plan *plan, u64 *f, u64 fstride, const u32 *src32,
                         u64 sstride32, u64 nchunks, u64 xor0, int batch, cudaStream_t st);
int fft_run_batch(const gf2e_fft_plan *plan, bool forward, u64 *f, u64 fstride, int batch,
                  cudaStream_t st);
int overlap_add_batch(const u64 *F, u64 fstride, u64 nchunks, u64 *out, u64 ostride, u64 ow,
                      int batch, cudaStream_t st);
int pointwise(u64 *fa, const u64 *fb, u64 n, cudaStream_t st);
int mul_fft_m(u64 abits, u64 bbits);
gf2e_fft_plan *cached_plan(int m);
u64 fft_plan_n(const gf2e_fft_plan *plan);
}  // namespace gf2e

namespace {

// ------------------------------------------------------------------------
// small-polynomial arithmetic on the host (the gcd of a hit is small)
typedef std::vector<u64> Poly;

long long pdeg(const Poly &a) {
    for (size_t i = a.size(); i-- > 0;)
        if (a[i]) return (long long)(i * 64 + 63 - __builtin_clzll(a[i]));
    return -1;
}
void ptrim(Poly &a) {
    while (!a.empty() && !a.back()) a.pop_back();
}
// a ^= b << sh
void pxor_shift(Poly &a, const Poly &b, u64 sh) {
    size_t ws = (size_t)(sh >> 6);
    unsigned bs = (unsigned)(sh & 63);
    if (a.size() < b.size() + ws + 1) a.resize(b.size() + ws + 1, 0);
    for (size_t j = 0; j < b.size(); j++) {
        a[j + ws] ^= b[j] << bs;
        if (bs) a[j + ws + 1] ^= b[j] >> (64 - bs);
    }
}
// a mod m
void pmod(Poly &a, const Poly &m) {
    long long dm = pdeg(m), da = pdeg(a);
    while (da >= dm) {
        pxor_shift(a, m, (u64)(da - dm));
        da = pdeg(a);
    }
    ptrim(a);
}
Poly psqr(const Poly &a) {
    Poly c(2 * a.size() + 1, 0);
    for (size_t i = 0; i < a.size(); i++)
        for (int h = 0; h < 2; h++) {
            u64 x = (a[i] >> (32 * h)) & 0xFFFFFFFFull;
            x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
            x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
            x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
            x = (x | (x << 2)) & 0x3333333333333333ull;
            x = (x | (x << 1)) & 0x5555555555555555ull;
            c[2 * i + h] ^= x;
        }
    ptrim(c);
    return c;
}
Poly pgcd(Poly a, Poly b) {
    ptrim(a);
    ptrim(b);
    while (!b.empty()) {
        pmod(a, b);
        std::swap(a, b);
    }
    return a;
}
bool pless(const Poly &x, const Poly &y) {
    size_t n = std::max(x.size(), y.size());
    for (size_t i = n; i-- > 0;) {
        u64 xv = i < x.size() ? x[i] : 0, yv = i < y.size() ? y[i] : 0;
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

// split g (product of distinct irreducibles of degree d) into its factors
// by the trace map: for random u, Tr(u) = u + u^2 + ... + u^(2^(d-1)) mod g is
// 0 or 1 modulo each factor, so gcd(Tr(u), g) splits g about half the time
void edf_split(const Poly &g, u64 d, u64 &rng, std::vector<Poly> &out, int depth = 0) {
    long long dg = pdeg(g);
    if (dg <= 0) return;
    if ((u64)dg == d || depth > 200) { out.push_back(g); return; }
    for (int tries = 0; tries < 64; tries++) {
        Poly u((size_t)(dg / 64) + 1, 0);
        for (auto &w : u) w = rng_next(rng);
        if (dg % 64 != 63) u.back() &= (1ull << (dg % 64 + 1)) - 1;
        pmod(u, g);
        Poly t = u, acc = u;
        for (u64 i = 1; i < d; i++) {
            t = psqr(t);
            pmod(t, g);
            if (acc.size() < t.size()) acc.resize(t.size(), 0);
            for (size_t j = 0; j < t.size(); j++) acc[j] ^= t[j];
        }
        ptrim(acc);
        Poly h = pgcd(g, acc);
        long long dh = pdeg(h);
        if (dh > 0 && dh < dg) {
            Poly q = g, h2 = h;
            // g / h by long division
            Poly quo((size_t)((dg - dh) / 64) + 1, 0);
            Poly rem = g;
            long long dr = pdeg(rem);
            while (dr >= dh) {
                u64 sh = (u64)(dr - dh);
                quo[sh >> 6] |= 1ull << (sh & 63);
                pxor_shift(rem, h2, sh);
                dr = pdeg(rem);
            }
            ptrim(quo);
            edf_split(h, d, rng, out, depth + 1);
            edf_split(quo, d, rng, out, depth + 1);
            return;
        }
    }
    out.push_back(g);           // not split: reported as is (caller checks degree)
}

}  // namespace

namespace gf2e {

// least k in [kmin, kmax] with gcd(x^(2^k) + x, g) != 1, and the numerically
// least irreducible factor of that degree; false if none
bool resolve_factor(const Poly &g_in, u64 kmin, u64 kmax, u64 &d_out, Poly &mask) {
    Poly g = g_in;
    ptrim(g);
    long long dg = pdeg(g);
    if (dg <= 0) return false;
    Poly h{2};                               // x mod g
    pmod(h, g);
    // every k from 1 is checked: the first k with a non-trivial gcd is the
    // least factor degree of g even when g also holds factors below kmin
    // (input that was not a genuine survivor, which the reference reports
    // with a warning, trinomial_scan.cu:288-296)
    (void)kmin;
    for (u64 k = 1; k <= kmax; k++) {
        h = psqr(h);
        pmod(h, g);
        Poly hx = h;
        if (hx.empty()) hx.push_back(0);
        hx[0] ^= 2;
        ptrim(hx);
        Poly gk = pgcd(g, hx);
        long long dk = pdeg(gk);
        if (dk > 0) {
            d_out = k;
            if ((u64)dk == k) { mask = gk; return true; }
            std::vector<Poly> parts;
            u64 rng = 0x243F6A8885A308D3ull ^ k;
            edf_split(gk, k, rng, parts);
            bool have = false;
            for (auto &p : parts) {
                if ((u64)pdeg(p) != k) return false;
                if (!have || pless(p, mask)) { mask = p; have = true; }
            }
            return have;
        }
    }
    return false;
}

}  // namespace gf2e

extern "C" {

int gf2e_resolve_factor(const uint64_t *g_host, size_t gw, uint64_t kmin, uint64_t kmax,
                        uint64_t *d_out, uint64_t *mask_host, size_t mask_cap_words,
                        size_t *mask_words) {
    if (!g_host || !d_out || !mask_host || !mask_words) return gf2e::invalid("null argument");
    Poly g(g_host, g_host + gw), mask;
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
