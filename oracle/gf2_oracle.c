/*
 * gf2_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference algorithms on the hot path, used as the
 * parity checker for the CUDA engine.  Nothing in the product library links
 * or calls this file; only tests, the smoke check and bench.py's CPU-baseline
 * leg load it (through oracle/oracle.py).
 *
 * Every function cites the reference file:line it restates (paths are within
 * the reference project).  The arithmetic follows the reference step for
 * step where the result depends on a choice (primitive-polynomial search
 * order, the Cantor-basis solution with zero constant term, the transform's
 * point order); elsewhere it is plain textbook GF(2) arithmetic.
 *
 * Pinning: tests/test_oracle.py checks these functions against golden
 * vectors produced by the reference itself (sieve_ref, cantor_ref's
 * gf2x_fft_mul, the reference kernels of trinomial_stage2 / trinomial_scan
 * run through the reference's CPU emulation header) and against the
 * reference's own known-answer tests.
 *
 * Bit layout everywhere: little-endian u64 words, bit i of word w is the
 * coefficient of x^(64w+i) (gf2_gcd.h:1-4).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t u64;
typedef uint32_t u32;

#if defined(__x86_64__)
#include <immintrin.h>
#define ORC_HAVE_X86 1
#endif

/* ======================================================================
 * GF(2^d), d <= 32, elements as u32, modulus q as u64 with bit d set.
 * Follows gf2_small_field.h:30-135.
 * ====================================================================== */
static u64 clmul32(u32 a, u32 b) {
    u64 r = 0, x = a;
    while (b) {
        if (b & 1u) r ^= x;
        x <<= 1;
        b >>= 1;
    }
    return r;
}

/* gf2_small_field.h:57-64 */
static u32 gf_reduce(u64 t, u64 q, int d) {
    for (int b = 2 * d - 2; b >= d; b--)
        if ((t >> b) & 1u) t ^= q << (b - d);
    return (u32)t;
}

u32 orc_gf_mul(u32 a, u32 b, u64 q, int d) { return gf_reduce(clmul32(a, b), q, d); }

/* gf2_small_field.h:74-78 */
u32 orc_gf_mulx(u32 a, u64 q, int d) {
    u64 t = (u64)a << 1;
    if ((t >> d) & 1u) t ^= q;
    return (u32)t;
}

/* gf2_small_field.h:81-88 (any correct exponentiation gives the same value) */
u32 orc_gf_pow(u32 base, u64 e, u64 q, int d) {
    u32 r = 1, b = base;
    while (e) {
        if (e & 1u) r = orc_gf_mul(r, b, q, d);
        b = orc_gf_mul(b, b, q, d);
        e >>= 1;
    }
    return r;
}

static u64 gcd64(u64 a, u64 b) {
    while (b) { u64 t = a % b; a = b; b = t; }
    return a;
}

/* modular inverse, gf2_small_field.h:101-111 */
static u64 invmod64(u64 a, u64 m) {
    int64_t t = 0, nt = 1, rr = (int64_t)m, nr = (int64_t)(a % m);
    while (nr) {
        int64_t qq = rr / nr, tmp;
        tmp = t - qq * nt; t = nt; nt = tmp;
        tmp = rr - qq * nr; rr = nr; nr = tmp;
    }
    if (t < 0) t += (int64_t)m;
    return (u64)t;
}

/* distinct prime factors by trial division, gf2_field_setup.h:14-21 */
static int prime_factors(u64 m, u64 *out) {
    int n = 0;
    for (u64 p = 2; p * p <= m; p += (p == 2 ? 1 : 2)) {
        if (m % p == 0) {
            out[n++] = p;
            while (m % p == 0) m /= p;
        }
    }
    if (m > 1) out[n++] = m;
    return n;
}

/* gf2_field_setup.h:25-34 */
int orc_is_irreducible(u64 q, int d) {
    u32 chain[65];
    u32 t = 2;
    chain[0] = t;
    for (int i = 1; i <= d; i++) { t = orc_gf_mul(t, t, q, d); chain[i] = t; }
    if (chain[d] != 2) return 0;
    u64 ps[16];
    int np = prime_factors((u64)d, ps);
    for (int i = 0; i < np; i++)
        if (chain[d / ps[i]] == 2) return 0;
    return 1;
}

/* gf2_field_setup.h:37-41 */
static int x_is_primitive(u64 q, int d, u64 M) {
    u64 ps[64];
    int np = prime_factors(M, ps);
    for (int i = 0; i < np; i++)
        if (orc_gf_pow(2, M / ps[i], q, d) == 1) return 0;
    return 1;
}

/* smallest primitive polynomial of degree d (ascending odd candidates),
 * gf2_field_setup.h:49-58.  Returns 0 if none (cannot happen). */
u64 orc_find_primitive_poly(int d) {
    u64 M = ((u64)1 << d) - 1;
    for (u64 q = ((u64)1 << d) | 1u; q < ((u64)2 << d); q += 2)
        if (orc_is_irreducible(q, d) && x_is_primitive(q, d, M)) return q;
    return 0;
}

/* minimal polynomial of g^j as the product of (x + conjugate),
 * gf2_small_field.h:117-135.  Returns the (d+1)-bit mask or 0. */
static u64 minpoly_product(u32 j, int d, u32 M, u64 q, const u32 *A) {
    u32 P[64];
    for (int k = 0; k <= d; k++) P[k] = 0;
    P[0] = 1;
    u32 rt = j;
    for (int i = 0; i < d; i++) {
        u32 root = A[rt];
        for (int k = i + 1; k >= 1; k--) P[k] = P[k - 1] ^ orc_gf_mul(root, P[k], q, d);
        P[0] = orc_gf_mul(root, P[0], q, d);
        rt = ((rt << 1) | (rt >> (d - 1))) & M;
    }
    u64 mask = 0;
    for (int k = 0; k <= d; k++) {
        if (P[k] > 1) return 0;
        mask |= (u64)P[k] << k;
    }
    return mask;
}

/* ======================================================================
 * Zech-log sieve, sieve_ref.cpp:58-134.
 * best has smax+1 entries; key = (d << 48) | mask, min over keys.
 * If init != 0, best[] is first set to all-ones.  Degrees dmin..dmax.
 * Returns 0, or -d if gcd(r, 2^d - 1) != 1 at degree d (sieve_ref.cpp:79-83).
 * Optional per-degree statistics: classes[d], marks[d] (arrays of >= dmax+1).
 * ====================================================================== */
int orc_sieve(u64 r, int dmin, int dmax, u64 smax, u64 *best, int init,
              u64 *classes_out, u64 *marks_out) {
    if (init)
        for (u64 s = 0; s <= smax; s++) best[s] = ~(u64)0;
    for (int d = dmin; d <= dmax; d++) {
        const u64 M = ((u64)1 << d) - 1;
        const u64 q = orc_find_primitive_poly(d);
        u64 subq[16], ps[16];
        int np = prime_factors((u64)d, ps);
        for (int i = 0; i < np; i++) subq[i] = M / (((u64)1 << (d / ps[i])) - 1);
        const u64 rmod = r % M;
        if (gcd64(rmod ? rmod : M, M) != 1) return -d;
        u32 *A = (u32 *)malloc(sizeof(u32) * M);
        u32 *L = (u32 *)malloc(sizeof(u32) * (M + 1));
        u32 t = 1;
        for (u64 i = 0; i < M; i++) { A[i] = t; t = orc_gf_mulx(t, q, d); }
        for (u64 i = 0; i < M; i++) L[A[i]] = (u32)i;
        u64 nclass = 0, nmark = 0;
        for (u64 j = 1; j < M; j++) {
            int skip = 0;
            for (int i = 0; i < np; i++)
                if (j % subq[i] == 0) { skip = 1; break; }
            if (skip) continue;
            u64 jj = j;
            int minimal = 1;
            for (int i = 1; i < d; i++) {
                jj = ((jj << 1) | (jj >> (d - 1))) & M;
                if (jj < j) { minimal = 0; break; }
            }
            if (!minimal) continue;
            nclass++;
            u64 u = (j * rmod) % M;
            if (u == 0) continue;
            u64 v = L[A[u] ^ 1u];
            u64 gg = gcd64(j, M);
            if (v % gg) continue;
            u64 n = M / gg;
            u64 s0 = (invmod64(j / gg, n) * (v / gg)) % n;
            u64 mask = minpoly_product((u32)j, d, (u32)M, q, A);
            if (!mask) { free(A); free(L); return -1000 - d; }
            u64 key = ((u64)d << 48) | mask;
            for (u64 s = (s0 ? s0 : n); s <= smax; s += n) {
                nmark++;
                if (key < best[s]) best[s] = key;
            }
        }
        if (classes_out) classes_out[d] = nclass;
        if (marks_out) marks_out[d] = nmark;
        free(A);
        free(L);
    }
    return 0;
}

/* independent brute force, sieve_ref.cpp:142-160 */
void orc_sieve_brute(u64 r, int depth, u64 smax, u64 *best) {
    for (u64 s = 0; s <= smax; s++) best[s] = ~(u64)0;
    for (int d = 2; d <= depth; d++) {
        for (u64 m = ((u64)1 << d) | 1u; m < ((u64)2 << d); m += 2) {
            if (!orc_is_irreducible(m, d)) continue;
            u32 xr = orc_gf_pow(2, r, m, d);
            u32 xs = 1;
            u64 key = ((u64)d << 48) | m;
            for (u64 s = 1; s <= smax; s++) {
                xs = orc_gf_mulx(xs, m, d);
                if ((xr ^ xs ^ 1u) == 0 && key < best[s]) best[s] = key;
            }
        }
    }
}

/* ======================================================================
 * GF(2)[x]/(x^r + x^s + 1): squaring by bit-spread and two fold passes.
 * Restates gf2_trinomial_cuda.h:22-74 and TrinGPU::reduce/square_A
 * (gf2_trinomial_cuda.h:136-154).
 * ====================================================================== */
static u64 spread32(u32 v) {
    u64 x = v;
    x = (x | (x << 16)) & 0x0000FFFF0000FFFFULL;
    x = (x | (x << 8)) & 0x00FF00FF00FF00FFULL;
    x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0FULL;
    x = (x | (x << 2)) & 0x3333333333333333ULL;
    x = (x | (x << 1)) & 0x5555555555555555ULL;
    return x;
}

static inline size_t words_of(u64 bits) { return (size_t)((bits + 63) >> 6); }

/* 64-bit window of src at bit pos, restricted to source bits in [lo,hi)
 * (gf2_trinomial_cuda.h:44-59) */
static u64 window64(const u64 *src, size_t nw, u64 pos, u64 lo, u64 hi) {
    size_t w0 = (size_t)(pos >> 6);
    unsigned sh = (unsigned)(pos & 63);
    u64 a = (w0 < nw) ? src[w0] : 0;
    u64 b = (w0 + 1 < nw) ? src[w0 + 1] : 0;
    u64 v = sh ? ((a >> sh) | (b << (64 - sh))) : a;
    u64 lc = (lo > pos) ? lo - pos : 0;
    u64 hc = (hi > pos) ? hi - pos : 0;
    if (lc >= 64 || hc == 0) return 0;
    if (hc > 64) hc = 64;
    u64 m = (hc >= 64) ? ~(u64)0 : (((u64)1 << hc) - 1);
    if (lc) m &= ~(((u64)1 << lc) - 1);
    return v & m;
}

/* one fold pass x^e -> x^(e-r) + x^(e-r+s) for e in [r,L)
 * (gf2_trinomial_cuda.h:63-74) */
static void fold_pass(const u64 *src, size_t snw, u64 *dst, size_t dnw,
                      u64 r, u64 s, u64 L) {
    for (size_t w = 0; w < dnw; w++) {
        u64 pos = (u64)w << 6;
        dst[w] = window64(src, snw, pos, 0, r) ^ window64(src, snw, pos + r, r, L) ^
                 window64(src, snw, pos + (r - s), r, L);
    }
}

/* reduce t0 (length L bits, 2*nw words, clobbered) mod T into out (nw words)
 * (gf2_trinomial_cuda.h:136-146) */
static void reduce_two_pass(u64 *t0, u64 *t1, size_t nw, u64 r, u64 s, u64 L,
                            u64 *out) {
    size_t nw2 = 2 * nw;
    fold_pass(t0, nw2, t1, nw2, r, s, L);
    u64 L2 = (L > r) ? (r + s - 1) : L;
    fold_pass(t1, nw2, t0, nw2, r, s, L2);
    memcpy(out, t0, nw * sizeof(u64));
}

/* out = in^2 mod (x^r + x^s + 1); out may alias in.  Returns 0 or -1 if s is
 * outside 1 <= s, 2s < r (gf2_trinomial_cuda.h:118-123). */
int orc_trin_square(const u64 *in, u64 *out, u64 r, u64 s) {
    if (!(s >= 1 && 2 * s < r)) return -1;
    size_t nw = words_of(r), nw2 = 2 * nw;
    u64 *t0 = (u64 *)malloc(nw2 * sizeof(u64));
    u64 *t1 = (u64 *)malloc(nw2 * sizeof(u64));
    for (size_t w = 0; w < nw2; w++) {
        u64 v = in[w >> 1];
        t0[w] = spread32((u32)((w & 1) ? (v >> 32) : v));
    }
    reduce_two_pass(t0, t1, nw, r, s, 2 * r - 1, out);
    free(t0);
    free(t1);
    return 0;
}

/* k squarings in place (state has words_of(r) words) */
int orc_trin_square_k(u64 *state, u64 r, u64 s, u64 k) {
    if (!(s >= 1 && 2 * s < r)) return -1;
    size_t nw = words_of(r), nw2 = 2 * nw;
    u64 *t0 = (u64 *)malloc(nw2 * sizeof(u64));
    u64 *t1 = (u64 *)malloc(nw2 * sizeof(u64));
    for (u64 it = 0; it < k; it++) {
        for (size_t w = 0; w < nw2; w++) {
            u64 v = state[w >> 1];
            t0[w] = spread32((u32)((w & 1) ? (v >> 32) : v));
        }
        reduce_two_pass(t0, t1, nw, r, s, 2 * r - 1, state);
    }
    free(t0);
    free(t1);
    return 0;
}

/* naive bit-serial reduction of v (bits < nbits) mod T, in place
 * (gf2_trinomial_cuda.h:182-190) */
void orc_mod_trinomial(u64 *v, u64 nbits, u64 r, u64 s) {
    for (u64 e = nbits; e-- > r;) {
        if (!((v[e >> 6] >> (e & 63)) & 1u)) continue;
        v[e >> 6] ^= (u64)1 << (e & 63);
        u64 e1 = e - r, e2 = e - r + s;
        v[e1 >> 6] ^= (u64)1 << (e1 & 63);
        v[e2 >> 6] ^= (u64)1 << (e2 & 63);
    }
}

/* naive bit-serial product, gf2_cantor_engine.h:247-260; out has
 * words_of(abits+bbits)+1 words */
void orc_naive_mul(const u64 *a, u64 abits, const u64 *b, u64 bbits, u64 *out) {
    size_t ow = words_of(abits + bbits) + 1, wb = words_of(bbits);
    memset(out, 0, ow * sizeof(u64));
    for (u64 i = 0; i < abits; i++) {
        if (!((a[i >> 6] >> (i & 63)) & 1u)) continue;
        size_t w = (size_t)(i >> 6), sh = (size_t)(i & 63);
        for (size_t j = 0; j < wb; j++) {
            u64 v = b[j];
            out[w + j] ^= v << sh;
            if (sh) out[w + j + 1] ^= v >> (64 - sh);
        }
    }
}

/* independent naive squaring mod T (gf2_trinomial_cuda.h:191-198) */
int orc_trin_square_naive(u64 *state, u64 r, u64 s) {
    if (!(s >= 1 && 2 * s < r)) return -1;
    size_t nw = words_of(r), ow = words_of(2 * r) + 1;
    u64 *sq = (u64 *)calloc(ow, sizeof(u64));
    orc_naive_mul(state, r, state, r, sq);
    orc_mod_trinomial(sq, 2 * r - 1, r, s);
    memcpy(state, sq, nw * sizeof(u64));
    free(sq);
    return 0;
}

/* ======================================================================
 * GF(2^64) = GF(2)[x]/(x^64+x^4+x^3+x+1) and the Cantor additive FFT.
 * Restates gf2_cantor_core.h:30-110 and gf2_cantor_engine.h:52-242.
 * ====================================================================== */

/* bit-serial field multiply, gf2_cantor_engine.h:52-61 */
u64 orc_gf64_mul_bitref(u64 a, u64 b) {
    u64 r = 0;
    while (b) {
        if (b & 1u) r ^= a;
        u64 hi = a >> 63;
        a = (a << 1) ^ (hi ? 0x1BULL : 0);
        b >>= 1;
    }
    return r;
}

typedef struct { u64 lo, hi; } orc128;

static orc128 clmul64_portable(u64 a, u64 b) {
    orc128 r = {0, 0};
    for (int i = 0; i < 64; i++)
        if ((b >> i) & 1u) {
            r.lo ^= a << i;
            if (i) r.hi ^= a >> (64 - i);
        }
    return r;
}

#ifdef ORC_HAVE_X86
__attribute__((target("pclmul,sse4.1"))) static orc128 clmul64_x86(u64 a, u64 b) {
    __m128i p = _mm_clmulepi64_si128(_mm_cvtsi64_si128((long long)a),
                                     _mm_cvtsi64_si128((long long)b), 0x00);
    orc128 r;
    r.lo = (u64)_mm_cvtsi128_si64(p);
    r.hi = (u64)_mm_extract_epi64(p, 1);
    return r;
}
static int g_have_pclmul = -1;
static orc128 clmul64(u64 a, u64 b) {
    if (g_have_pclmul < 0) {
        __builtin_cpu_init();
        g_have_pclmul = __builtin_cpu_supports("pclmul") && __builtin_cpu_supports("sse4.1");
    }
    return g_have_pclmul ? clmul64_x86(a, b) : clmul64_portable(a, b);
}
#else
static orc128 clmul64(u64 a, u64 b) { return clmul64_portable(a, b); }
#endif

/* reduction mod x^64 + x^4 + x^3 + x + 1 (gf2_cantor_core.h:60-66) */
static u64 gf64_reduce(orc128 t) {
    u64 h = t.hi;
    u64 lo = t.lo ^ h ^ (h << 1) ^ (h << 3) ^ (h << 4);
    u64 h2 = (h >> 63) ^ (h >> 61) ^ (h >> 60);
    return lo ^ h2 ^ (h2 << 1) ^ (h2 << 3) ^ (h2 << 4);
}

u64 orc_gf64_mul(u64 a, u64 b) { return gf64_reduce(clmul64(a, b)); }

/* Cantor basis b[0]=1, b[i]^2 + b[i] = b[i-1], each b[i] the solution of
 * y^2 + y = b[i-1] whose constant coefficient is 0 (this is the solution the
 * reference's pivoting picks: gf2_cantor_engine.h:78-103 never puts the
 * kernel vector 1 into a pivot combination).  Returns the chain length. */
int orc_cantor_basis(u64 *b) {
    /* row-reduce the 63 images T(x^i), i >= 1, keeping preimages */
    u64 piv_v[64], piv_t[64];
    memset(piv_v, 0, sizeof piv_v);
    memset(piv_t, 0, sizeof piv_t);
    for (int i = 1; i < 64; i++) {
        u64 e = (u64)1 << i;
        u64 v = orc_gf64_mul(e, e) ^ e, t = e;
        for (int bit = 63; bit >= 0 && v; bit--) {
            if (!((v >> bit) & 1u)) continue;
            if (piv_v[bit]) { v ^= piv_v[bit]; t ^= piv_t[bit]; }
            else { piv_v[bit] = v; piv_t[bit] = t; v = 0; }
        }
    }
    b[0] = 1;
    int len = 1;
    while (len < 64) {
        u64 c = b[len - 1], v = c, y = 0;
        int ok = 1;
        for (int bit = 63; bit >= 0 && v; bit--) {
            if (!((v >> bit) & 1u)) continue;
            if (!piv_v[bit]) { ok = 0; break; }
            v ^= piv_v[bit];
            y ^= piv_t[bit];
        }
        if (!ok || v) break;
        y &= ~(u64)1;                      /* the zero-constant solution */
        if ((orc_gf64_mul(y, y) ^ y) != c) {
            y ^= 1;
            if ((orc_gf64_mul(y, y) ^ y) != c) return -1;
        }
        b[len++] = y;
    }
    return len;
}

/* twiddles W[t] = XOR of b[j+1] over set bits j of t, t < n/2
 * (gf2_cantor_engine.h:130-139) */
void orc_fft_twiddles(int m, const u64 *basis, u64 *W) {
    size_t half = (size_t)1 << (m - 1);
    W[0] = 0;
    for (size_t t = 1; t < half; t++) {
        int hb = 63 - __builtin_clzll((u64)t);
        W[t] = W[t ^ ((size_t)1 << hb)] ^ basis[hb + 1];
    }
}

static void xr_range(u64 *f, size_t dst, size_t src, size_t len) {
    for (size_t k = 0; k < len; k++) f[dst + k] ^= f[src + k];
}

/* forward transform, gf2_cantor_engine.h:146-165 */
void orc_fft_fwd(u64 *f, int m, const u64 *W) {
    size_t n = (size_t)1 << m;
    for (int L = 0; L <= m - 2; L++) {
        size_t S = n >> L;
        for (size_t B = S; B >= 4; B >>= 1) {
            size_t q = B >> 2, h = B >> 1;
            for (size_t o = 0; o < S; o += B) {
                xr_range(f, (o + h) << L, (o + h + q) << L, q << L);
                xr_range(f, (o + q) << L, (o + h) << L, q << L);
            }
        }
    }
    for (int L = m - 1; L >= 0; L--) {
        size_t half = n >> 1, mask = ((size_t)1 << L) - 1;
        for (size_t p = 0; p < half; p++) {
            size_t t = p >> L, id = p & mask;
            size_t i1 = id + (t << (L + 1)), i2 = i1 + ((size_t)1 << L);
            u64 e = f[i1] ^ orc_gf64_mul(W[t], f[i2]);
            f[i1] = e;
            f[i2] = e ^ f[i2];
        }
    }
}

/* inverse transform, gf2_cantor_engine.h:168-187 */
void orc_fft_inv(u64 *f, int m, const u64 *W) {
    size_t n = (size_t)1 << m;
    for (int L = 0; L <= m - 1; L++) {
        size_t half = n >> 1, mask = ((size_t)1 << L) - 1;
        for (size_t p = 0; p < half; p++) {
            size_t t = p >> L, id = p & mask;
            size_t i1 = id + (t << (L + 1)), i2 = i1 + ((size_t)1 << L);
            u64 h = f[i1] ^ f[i2];
            f[i1] = f[i1] ^ orc_gf64_mul(W[t], h);
            f[i2] = h;
        }
    }
    for (int L = m - 2; L >= 0; L--) {
        size_t S = n >> L;
        for (size_t B = 4; B <= S; B <<= 1) {
            size_t q = B >> 2, h = B >> 1;
            for (size_t o = 0; o < S; o += B) {
                xr_range(f, (o + q) << L, (o + h) << L, q << L);
                xr_range(f, (o + h) << L, (o + h + q) << L, q << L);
            }
        }
    }
}

/* FFT size exponent for a product of abits x bbits: smallest m >= 1 with
 * 2^m >= ca + cb - 1 (gf2_cantor_engine.h:232-238) */
int orc_fft_m_for(u64 abits, u64 bbits) {
    u64 ca = (abits + 31) >> 5, cb = (bbits + 31) >> 5;
    int m = 1;
    while (((u64)1 << m) < ca + cb - 1) m++;
    return m;
}

/* full product via the transform, gf2_cantor_engine.h:207-242.
 * out has words_of(abits+bbits)+1 words and is fully overwritten. */
int orc_fft_mul(const u64 *a, u64 abits, const u64 *b, u64 bbits, u64 *out) {
    if (abits == 0 || bbits == 0) return -1;
    u64 basis[64];
    int blen = orc_cantor_basis(basis);
    int m = orc_fft_m_for(abits, bbits);
    if (blen < m) return -2;
    size_t n = (size_t)1 << m;
    u64 ca = (abits + 31) >> 5, cb = (bbits + 31) >> 5;
    size_t wa = words_of(abits), wb = words_of(bbits);
    u64 *W = (u64 *)malloc((n / 2 + 1) * sizeof(u64));
    u64 *FA = (u64 *)calloc(n, sizeof(u64));
    u64 *FB = (u64 *)calloc(n, sizeof(u64));
    orc_fft_twiddles(m, basis, W);
    for (u64 k = 0; k < ca; k++) {
        size_t w = (size_t)(k >> 1);
        FA[k] = (w < wa) ? (u32)(a[w] >> ((k & 1) * 32)) : 0;
    }
    for (u64 k = 0; k < cb; k++) {
        size_t w = (size_t)(k >> 1);
        FB[k] = (w < wb) ? (u32)(b[w] >> ((k & 1) * 32)) : 0;
    }
    orc_fft_fwd(FA, m, W);
    orc_fft_fwd(FB, m, W);
    for (size_t k = 0; k < n; k++) FA[k] = orc_gf64_mul(FA[k], FB[k]);
    orc_fft_inv(FA, m, W);
    size_t ow = words_of(abits + bbits) + 1;
    memset(out, 0, ow * sizeof(u64));
    for (u64 k = 0; k < ca + cb - 1; k++) {
        u64 e = FA[k];
        size_t pos = 32 * (size_t)k, w = pos >> 6, sh = pos & 63;
        out[w] ^= e << sh;
        if (sh) out[w + 1] ^= e >> 32;
    }
    free(W);
    free(FA);
    free(FB);
    return 0;
}

/* word-comb schoolbook with 64x64 carry-less products
 * (gf2_cantor_engine.h:263-274) */
void orc_comb_mul(const u64 *a, u64 abits, const u64 *b, u64 bbits, u64 *out) {
    size_t wa = words_of(abits), wb = words_of(bbits), ow = words_of(abits + bbits) + 1;
    memset(out, 0, ow * sizeof(u64));
    for (size_t i = 0; i < wa; i++)
        for (size_t j = 0; j < wb; j++) {
            orc128 p = clmul64(a[i], b[j]);
            out[i + j] ^= p.lo;
            out[i + j + 1] ^= p.hi;
        }
}

/* residue of a bit array mod an irreducible q of degree d <= 62
 * (ModP::residue, gf2_cantor_engine.h:278-325) */
static u64 modq_mul(u64 a, u64 b, u64 q, int d) {
    orc128 t = clmul64(a, b);
    for (int bit = 2 * d - 2; bit >= d; bit--) {
        u64 have = ((bit >= 64 ? t.hi : t.lo) >> (bit & 63)) & 1u;
        if (!have) continue;
        int sh = bit - d;
        t.lo ^= q << sh;
        if (sh) t.hi ^= q >> (64 - sh);
    }
    return t.lo;
}
static u64 modq_red64(u64 v, u64 q, int d) {
    for (int bit = 63; bit >= d; bit--)
        if ((v >> bit) & 1u) v ^= q << (bit - d);
    return v;
}
u64 orc_residue(const u64 *a, u64 abits, u64 q, int d) {
    size_t wa = words_of(abits);
    u64 x64 = 1, base = 2, e = 64;
    while (e) {
        if (e & 1u) x64 = modq_mul(x64, base, q, d);
        base = modq_mul(base, base, q, d);
        e >>= 1;
    }
    u64 r = 0;
    for (size_t w = wa; w-- > 0;) r = modq_mul(r, x64, q, d) ^ modq_red64(a[w], q, d);
    return r;
}
u64 orc_modq_mul(u64 a, u64 b, u64 q, int d) { return modq_mul(a, b, q, d); }

/* ======================================================================
 * General GF(2)[x] utilities: degree, gcd, divisibility, powmod.
 * Restates gf2_gcd.h:26-145 and check-ntl.c:17-58.
 * ====================================================================== */
int64_t orc_poly_deg(const u64 *w, size_t nw) {
    for (size_t i = nw; i-- > 0;)
        if (w[i]) return (int64_t)(i * 64 + 63 - __builtin_clzll(w[i]));
    return -1;
}

/* A ^= B << sh, B of degree bdeg (gf2_gcd.h:37-45) */
static void xor_shift(u64 *A, size_t an, const u64 *B, int64_t bdeg, u64 sh) {
    size_t ws = (size_t)(sh >> 6);
    unsigned bs = (unsigned)(sh & 63);
    size_t bw = (size_t)(bdeg >> 6) + 1;
    for (size_t j = bw; j-- > 0;) {
        u64 v = B[j];
        A[j + ws] ^= v << bs;
        if (bs && j + ws + 1 < an) A[j + ws + 1] ^= v >> (64 - bs);
    }
}

/* naive Euclid (gf2_gcd.h:48-75).  Returns deg(gcd) (0 for gcd == 1 or
 * gcd(0,0)); writes the gcd (g_cap words, zero-filled) if g != NULL. */
int64_t orc_poly_gcd(const u64 *a, size_t aw, const u64 *b, size_t bw, u64 *g,
                     size_t g_cap) {
    size_t nw = (aw > bw ? aw : bw) + 1;
    u64 *A = (u64 *)calloc(nw, sizeof(u64));
    u64 *B = (u64 *)calloc(nw, sizeof(u64));
    if (aw) memcpy(A, a, aw * sizeof(u64));
    if (bw) memcpy(B, b, bw * sizeof(u64));
    int64_t da = orc_poly_deg(A, nw), db = orc_poly_deg(B, nw);
    if (da < db) { u64 *t = A; A = B; B = t; int64_t x = da; da = db; db = x; }
    while (db >= 0) {
        while (da >= db) {
            xor_shift(A, nw, B, db, (u64)(da - db));
            da = orc_poly_deg(A, (size_t)(da >> 6) + 1);
            if (da < 0) break;
        }
        u64 *t = A; A = B; B = t;
        int64_t x = da; da = db; db = x;
    }
    int64_t res = da < 0 ? 0 : da;
    if (g) {
        memset(g, 0, g_cap * sizeof(u64));
        if (da >= 0) {
            size_t gw = (size_t)(da >> 6) + 1;
            memcpy(g, A, (gw < g_cap ? gw : g_cap) * sizeof(u64));
        }
    }
    free(A);
    free(B);
    return res;
}

/* a mod f in place (a has an words, f of degree df >= 0) */
static void poly_rem(u64 *a, size_t an, const u64 *f, int64_t df) {
    int64_t da = orc_poly_deg(a, an);
    while (da >= df) {
        xor_shift(a, an, f, df, (u64)(da - df));
        da = orc_poly_deg(a, (size_t)(da >> 6) + 1);
    }
}

/* x^e mod f into out (fw = words_of(df) words + 1 scratch handled inside) */
static void powx_mod(u64 e, const u64 *f, int64_t df, u64 *out, size_t fw) {
    size_t tw = 2 * fw + 2;
    u64 *t = (u64 *)calloc(tw, sizeof(u64));
    u64 *acc = (u64 *)calloc(fw + 1, sizeof(u64));
    acc[0] = 1;
    poly_rem(acc, fw + 1, f, df);
    int top = 63;
    while (top > 0 && !((e >> top) & 1u)) top--;
    for (int bit = top; bit >= 0; bit--) {
        /* square */
        memset(t, 0, tw * sizeof(u64));
        for (size_t w = 0; w < fw + 1; w++) {
            t[2 * w] ^= spread32((u32)acc[w]);
            t[2 * w + 1] ^= spread32((u32)(acc[w] >> 32));
        }
        poly_rem(t, tw, f, df);
        memcpy(acc, t, (fw + 1) * sizeof(u64));
        if ((e >> bit) & 1u) {
            /* multiply by x */
            u64 carry = 0;
            for (size_t w = 0; w < fw + 1; w++) {
                u64 nc = acc[w] >> 63;
                acc[w] = (acc[w] << 1) | carry;
                carry = nc;
            }
            poly_rem(acc, fw + 1, f, df);
        }
    }
    memcpy(out, acc, fw * sizeof(u64));
    free(t);
    free(acc);
}

/* check-ntl.c:17-58: does the polynomial f (words fw, degree must be d)
 * divide x^r + x^s + 1?  Returns 1 yes, 0 no, -1 degree mismatch. */
int orc_factor_divides(u64 r, u64 s, u64 d, const u64 *f, size_t fw) {
    int64_t df = orc_poly_deg(f, fw);
    if (df != (int64_t)d || df < 1) return -1;
    size_t nw = (size_t)(df >> 6) + 1;
    u64 *xr = (u64 *)calloc(nw + 1, sizeof(u64));
    u64 *xs = (u64 *)calloc(nw + 1, sizeof(u64));
    powx_mod(r, f, df, xr, nw);
    powx_mod(s, f, df, xs, nw);
    xr[0] ^= 1;
    int ok = 1;
    for (size_t w = 0; w < nw; w++)
        if (xr[w] != xs[w]) { ok = 0; break; }
    free(xr);
    free(xs);
    return ok;
}

/* does m divide g (gf2_gcd.h:78-83) */
static int poly_divides(const u64 *m, size_t mw, const u64 *g, size_t gw) {
    int64_t dm = orc_poly_deg(m, mw);
    if (dm <= 0) return 0;
    size_t cap = (mw > gw ? mw : gw) + 1;
    u64 *t = (u64 *)calloc(cap, sizeof(u64));
    int64_t dd = orc_poly_gcd(m, mw, g, gw, t, cap);
    free(t);
    return dd == dm;
}

/* least degree-`target` divisor of g by ascending odd masks
 * (gf2_gcd.h:137-145).  Returns the mask or 0. */
u64 orc_edf_least_enum(const u64 *g, size_t gw, u64 target) {
    if (target > 22) return 0;
    for (u64 m = ((u64)1 << target) | 1u; m < ((u64)2 << target); m += 2)
        if (poly_divides(&m, 1, g, gw)) return m;
    return 0;
}

/* per-degree naive-gcd scan oracle (trinomial_scan.cu:393-421).
 * Result codes: 0 = not a survivor (factor of degree <= k0),
 *               1 = found (d, gdeg, g words, mask words if resolved),
 *               2 = "u" (no factor of degree <= maxd).
 * g and mask buffers have cap words; *mask_ok tells whether mask holds the
 * least factor (exact when gdeg == d, else by enumeration for d <= 22). */
int orc_scan_one(u64 r, u64 s, u64 k0, u64 maxd, u64 *d_out, u64 *gdeg_out,
                 u64 *g, u64 *mask, size_t cap, int *mask_ok) {
    size_t nw = words_of(r), tw = words_of(r + 1);
    u64 *T = (u64 *)calloc(tw, sizeof(u64));
    T[0] |= 1;
    T[s >> 6] |= (u64)1 << (s & 63);
    T[r >> 6] |= (u64)1 << (r & 63);
    u64 *F = (u64 *)calloc(nw, sizeof(u64));
    u64 *Fx = (u64 *)calloc(nw, sizeof(u64));
    u64 *gg = (u64 *)calloc(tw + 1, sizeof(u64));
    F[0] = 2;
    int res = 2;
    *mask_ok = 0;
    for (u64 k = 1; k <= maxd; k++) {
        orc_trin_square_k(F, r, s, 1);
        memcpy(Fx, F, nw * sizeof(u64));
        Fx[0] ^= 2;
        int64_t gd = orc_poly_gcd(Fx, nw, T, tw, gg, tw + 1);
        if (gd > 0) {
            if (k <= k0) { res = 0; break; }
            res = 1;
            *d_out = k;
            *gdeg_out = (u64)gd;
            size_t gw = (size_t)(gd >> 6) + 1;
            memset(g, 0, cap * sizeof(u64));
            memcpy(g, gg, (gw < cap ? gw : cap) * sizeof(u64));
            memset(mask, 0, cap * sizeof(u64));
            if ((u64)gd == k) {
                memcpy(mask, gg, (gw < cap ? gw : cap) * sizeof(u64));
                *mask_ok = 1;
            } else {
                u64 m = orc_edf_least_enum(gg, gw, k);
                if (m) { mask[0] = m; *mask_ok = 1; }
            }
            break;
        }
    }
    free(T);
    free(F);
    free(Fx);
    free(gg);
    return res;
}

/* lowercase hex of a polynomial, no leading zeros (gf2_gcd.h:96-105);
 * returns the number of characters written (buf must hold deg/4+2). */
int orc_poly_hex(const u64 *v, size_t nw, char *buf) {
    int64_t d = orc_poly_deg(v, nw);
    if (d < 0) { buf[0] = '0'; buf[1] = 0; return 1; }
    int k = 0;
    for (int64_t n = d / 4; n >= 0; n--) {
        unsigned dig = (unsigned)((v[(size_t)(n >> 4)] >> ((n & 15) * 4)) & 0xF);
        buf[k++] = "0123456789abcdef"[dig];
    }
    buf[k] = 0;
    return k;
}
