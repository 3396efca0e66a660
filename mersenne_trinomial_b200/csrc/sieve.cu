// sieve.cu -- Zech-log sieve for the smallest irreducible factor of degree
// d <= 40 of x^r + x^s + 1, for every s in [1, smax] at once.
//
// Degrees up to 31 keep every field element and modulus in 32 bits and use
// dense antilog and log tables (2 x 8 GB at d = 31, resident in HBM).  The
// reference switches to bucketed low-memory tables beyond its GPU memory
// (coarse_sieve.cu:920-1117, 64-bit fields of gf2_wide_field.h for d >= 33).
// Degrees 32..40 here ("wide") keep elements in 64 bits and store only the
// log table, as slices of the value range [lo, hi) sized to the workspace
// (one slice of 2^d entries when it fits: d = 32 takes 16 GB, d = 33 64 GB):
//   k_wide_leaders  once per degree: per coset leader j, x^(j r) + 1 by
//                   square-and-multiply-by-x (no antilog table), written
//                   with j to a leader list
//   k_wide_slice    walks the exponents with a multiply-by-x chain and
//                   writes L[v - lo] = i for the values x^i in the slice
//   k_wide_match    the list entries whose lookup lies in the slice: the
//                   same progression and minimal polynomial as the dense path
// so a degree costs one pass over j and one exponent walk per slice.  When
// the list does not fit the budget (d >= 38 by default) every slice redoes
// the pass over j (k_wide_classes).
//
// Number theory (the reference's, sieve_ref.cpp:8-26): in GF(2^d) built on
// the smallest primitive q_d (x generates the group of order M = 2^d - 1), an
// irreducible p of degree d with root beta = x^j divides x^r + x^s + 1 iff
// j*s == Z(j*r mod M) (mod M), Z the Zech logarithm Z(u) = log(x^u + 1): an
// arithmetic progression in s of modulus n = M / gcd(j, M).  Only the
// smallest j of each cyclotomic coset and no proper-subfield j is used;
// key (d << 48) | mask(p) is merged into best[s] with min.
//
// B200 mapping:
//   k_tables    antilog A[i] = x^i (a multiply-by-x chain per 32 entries) and
//               the log scatter L[A[i]] = i in the same pass (tables are
//               L2-resident up to d = 23: 2 x 32 MB, 2 x 8 GB at d = 31).
//   k_classes   one thread per j: coset/subfield filters, Zech lookup,
//               progression; the minimal polynomial only for classes that
//               mark some s <= smax, by GF(2) elimination on the powers
//               beta^0..beta^d (O(d^2) word ops instead of O(d^2) field
//               multiplies; the minimal polynomial is unique so the mask is
//               identical).  Progressions are routed by length:
//                 n < strip width    -> strip list (applied in shared memory)
//                 <= INLINE marks    -> marked at once with atomicMin
//                 otherwise          -> heavy list (grid-stride atomicMin)
//   k_heavy     all heavy progressions of all degrees, one launch.
//   k_strip     each CTA owns a strip-wide slice of best[], applies every
//               short-period progression with shared-memory atomics and
//               writes the slice back once (last writer, so plain min).
// All degrees are enqueued on one stream with no host round trip; the only
// synchronisation is the final overflow/status read.  A progression that
// finds the strip or heavy list full is marked inline by its class thread
// (same marks, so the same best[]; only slower).
#include "gf2e_internal.cuh"

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <mutex>
#include <vector>

namespace {

constexpr int DMAX = 31;                  // dense tables (32-bit elements)
constexpr int DMAX_WIDE = 40;             // 64-bit elements, sliced log table
constexpr int STRIP_LOG_MAX = 14;         // strip CTAs own 2^10..2^14 entries of best[]
                                          // (8..128 KB of shared memory), tunable
constexpr u64 INLINE = 32;                // marks done inline by the class thread
constexpr u64 SCAP = 1ull << 17;          // strip-list capacity
constexpr u64 HCAP = 1ull << 21;          // heavy-list capacity

struct Prog { u64 s0, n, key; };          // first s, period, packed key

struct Counters {
    unsigned long long nstrip, nheavy, overflow, bad;
    unsigned long long classes[DMAX_WIDE + 1];
    unsigned long long marks[DMAX_WIDE + 1];
    unsigned long long nlist;             // wide leader list fill
    unsigned long long spilled;           // progressions marked inline for want of list room
};

// List capacities in force: the workspace holds SCAP / HCAP records, and
// GF2E_SIEVE_STRIP_CAP / GF2E_SIEVE_HEAVY_CAP may lower them (tests use tiny
// ones to drive every progression through the spill path).
struct ListCaps {
    u64 strip, heavy;
};

// A progression that finds its list full is marked at once by the thread
// that found it: the same atomicMin marks the list kernels would make, so
// the result is unchanged, only slower.
GF2E_DEV void mark_inline(u64 first, u64 n, u64 smax, unsigned long long key,
                          unsigned long long *__restrict__ best) {
    for (u64 s = first; s <= smax; s += n) atomicMin(&best[s], key);
}

// workspace: progression lists and counters first, then the table region
// (dense A and L tables, or the wide log-table slice), whose size may be
// anything the caller provides above the minimum
struct Layout {
    size_t off_strip, off_heavy, off_cnt, off_region;
};

constexpr Layout layout() {
    return Layout{0, SCAP * sizeof(Prog), SCAP * sizeof(Prog) + HCAP * sizeof(Prog),
                  ((SCAP + HCAP) * sizeof(Prog) + sizeof(Counters) + 255) & ~(size_t)255};
}

size_t dense_table_bytes(int d) {
    size_t tab = ((size_t)1 << d) * sizeof(u32);
    return (tab + 255) & ~(size_t)255;
}

ListCaps list_caps() {
    auto cap = [](const char *name, u64 full) {
        const char *e = getenv(name);
        if (!e) return full;
        const unsigned long long v = strtoull(e, nullptr, 10);
        return (u64)std::min<unsigned long long>(std::max<unsigned long long>(v, 1), full);
    };
    return ListCaps{cap("GF2E_SIEVE_STRIP_CAP", SCAP), cap("GF2E_SIEVE_HEAVY_CAP", HCAP)};
}

// log-table entry bytes of a wide degree (exponents below 2^d)
size_t wide_entry_bytes(int d) { return d <= 32 ? 4 : 8; }

// default wide slice budget (GF2E_SIEVE_WIDE_GB overrides)
size_t wide_budget() {
    const char *e = getenv("GF2E_SIEVE_WIDE_GB");
    double gb = e ? atof(e) : 64.0;
    if (!(gb >= 0.25)) gb = 0.25;
    return (size_t)(gb * (double)(1ull << 30)) & ~(size_t)255;
}

// first degree sieved on the wide path (DMAX + 1; GF2E_SIEVE_WIDE_FROM
// lowers it, down to 8, so the two paths can be compared on the same degrees)
int wide_from() {
    const char *e = getenv("GF2E_SIEVE_WIDE_FROM");
    int v = e ? atoi(e) : DMAX + 1;
    return std::min(std::max(v, 8), DMAX + 1);
}

// table region a run of dmin..dmax needs at least / would like
size_t region_min(int dmin, int dmax) {
    const int w = wide_from();
    size_t need = dmin < w ? 2 * dense_table_bytes(std::min(dmax, w - 1)) : 0;
    if (dmax >= w) need = std::max<size_t>(need, (size_t)1 << 28);
    return need;
}
// number of irreducible polynomials of degree d over GF(2) (the coset
// leaders of degree d): (1/d) sum over k | d of mu(d/k) 2^k
u64 irreducible_count(int d) {
    long long sum = 0;
    for (int k = 1; k <= d; k++) {
        if (d % k) continue;
        int n = d / k, mu = 1;
        for (int p = 2; p <= n; p++) {
            if (n % p) continue;
            n /= p;
            if (n % p == 0) { mu = 0; break; }
            mu = -mu;
        }
        sum += mu * (long long)(1ull << k);
    }
    return (u64)(sum / d);
}

// wide leader list: (j, x^(j r) + 1) per coset leader, 16 bytes each; used
// when it fits in the slice budget (d <= 37 by default)
size_t leader_list_bytes(int d) { return ((size_t)irreducible_count(d) * 16 + 255) & ~(size_t)255; }
bool leader_list_wanted(int d) { return leader_list_bytes(d) <= wide_budget(); }

size_t region_want(int dmin, int dmax) {
    size_t want = region_min(dmin, dmax);
    if (dmax >= wide_from()) {
        size_t w = std::min(((size_t)1 << dmax) * wide_entry_bytes(dmax), wide_budget());
        if (leader_list_wanted(dmax)) w += leader_list_bytes(dmax);
        want = std::max(want, w);
    }
    return want;
}

// ---- small field GF(2^d), d <= 31, modulus q (bit d set)
GF2E_DEV u32 sf_mul(u32 a, u32 b, u32 q, int d) {
    u64 t = clmul32(a, b);
    for (int bit = 2 * d - 2; bit >= d; bit--)
        if ((t >> bit) & 1) t ^= (u64)q << (bit - d);
    return (u32)t;
}
GF2E_DEV u32 sf_mulx(u32 a, u32 q, int d) {
    u32 t = a << 1;
    return ((t >> d) & 1) ? (t ^ q) : t;
}
GF2E_DEV u32 sf_powx(u64 e, u32 q, int d) {     // x^e
    u32 r = 1, b = 2;
    while (e) {
        if (e & 1) r = sf_mul(r, b, q, d);
        b = sf_mul(b, b, q, d);
        e >>= 1;
    }
    return r;
}
// x mod (2^d - 1)
GF2E_DEV u64 mod_mersenne(u64 x, int d, u64 M) {
    while (x > M) x = (x & M) + (x >> d);
    return x == M ? 0 : x;
}
// gcd(a, m) for 1 <= a and m >= 2 by the extended Euclidean algorithm; when
// the gcd is 1, *inv = a^-1 mod m.  One division per step, about
// 0.84 ln(m) steps (fewer instructions and less divergence than the
// shift-and-subtract form on these sizes)
GF2E_DEV u64 gcd_inv(u64 a, u64 m, u64 *inv) {
    long long t = 0, nt = 1;
    u64 r = m, nr = a % m;
    while (nr) {
        const u64 q = r / nr;
        const long long tmp = t - (long long)q * nt;
        t = nt;
        nt = tmp;
        const u64 rr = r - q * nr;
        r = nr;
        nr = rr;
    }
    if (t < 0) t += (long long)m;
    *inv = (u64)t;
    return r;
}

// first s >= 1 of the progression j*s = v (mod M), M = 2^d - 1, and its
// period n; false when no s exists.  gcd(j, M) = 1 for almost every j, and
// then the inverse and the product are taken modulo the Mersenne number
GF2E_DEV bool progression(u64 j, u64 v, int d, u64 M, u64 &first, u64 &n) {
    u64 inv;
    const u64 gg = gcd_inv(j, M, &inv);
    u64 s0;
    if (gg == 1) {
        n = M;
        u64 p = 0;
        {
            unsigned __int128 t = (unsigned __int128)inv * v;
            while (t > M) t = (t & M) + (t >> d);
            p = t == M ? 0 : (u64)t;
        }
        s0 = p;
    } else {
        if (v % gg) return false;
        n = M / gg;
        u64 inv2;
        gcd_inv(j / gg, n, &inv2);                // coprime after dividing out gg
        s0 = (u64)(((unsigned __int128)inv2 * (v / gg)) % n);
    }
    first = s0 ? s0 : n;
    return true;
}

__global__ void k_tables(u32 *__restrict__ A, u32 *__restrict__ L, int d, u32 q, u64 M) {
    u64 nchunk = (M + 31) >> 5;
    for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < nchunk;
         t += (u64)gridDim.x * blockDim.x) {
        u64 i0 = t << 5;
        u32 v = sf_powx(i0, q, d);
        for (int e = 0; e < 32; e++) {
            u64 i = i0 + e;
            if (i >= M) break;
            A[i] = v;
            L[v] = (u32)i;
            v = sf_mulx(v, q, d);
        }
    }
}

struct DegreeArgs {
    int d;
    u32 q;
    u64 M, rmod, smax;
    int nsub;
    u64 subq[6];
    u64 strip;                            // strip width (entries of best[] per CTA)
    ListCaps caps;
};

// j is the least element of its cyclotomic coset {j 2^i mod M}
GF2E_DEV bool coset_least(u64 j, int d, u64 M) {
    u64 jj = j;
    for (int i = 1; i < d; i++) {
        jj = ((jj << 1) | (jj >> (d - 1))) & M;
        if (jj < j) return false;
    }
    return true;
}

// Calls work(i, true) for every i in [begin, end) with pred(i), with full
// warps: each warp tests 32 consecutive i at a time and queues the selected
// ones in shared memory (wq: 64 entries per warp), running `work` on 32 of
// them whenever 32 are queued, so a rare, expensive path does not execute
// with one active lane per warp.  work(i, false) pads the final partial
// batch; every lane of the warp calls work together.
template <typename Pred, typename Work>
GF2E_DEV void for_each_selected(u64 begin, u64 end, u64 *wq, Pred &&pred, Work &&work) {
    const int lane = threadIdx.x & 31;
    const u64 gw = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const u64 nw = ((u64)gridDim.x * blockDim.x) >> 5;
    int qn = 0;
    for (u64 base = begin + gw * 32; base < end; base += nw * 32) {
        const u64 i = base + lane;
        const bool sel = i < end && pred(i);
        const unsigned b = __ballot_sync(0xffffffffu, sel);
        if (sel) wq[qn + __popc(b & ((1u << lane) - 1u))] = i;
        qn += __popc(b);
        __syncwarp();
        if (qn >= 32) {
            const u64 ii = wq[qn - 32 + lane];
            __syncwarp();
            qn -= 32;
            work(ii, true);
        }
    }
    const u64 ii = lane < qn ? wq[lane] : 0;
    work(ii, lane < qn);
}

// every coset leader j in [1, M) (about 1 in d of the j)
template <typename Work>
GF2E_DEV void for_each_leader(u64 M, int d, u64 *wq, Work &&work) {
    for_each_selected(1, M, wq, [&](u64 j) { return coset_least(j, d, M); }, work);
}

GF2E_DEV void add_stats(unsigned long long my_classes, unsigned long long my_marks, int d,
                        Counters *cnt) {
    for (int o = 16; o; o >>= 1) {
        my_classes += __shfl_down_sync(0xffffffffu, my_classes, o);
        my_marks += __shfl_down_sync(0xffffffffu, my_marks, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (my_classes) atomicAdd(&cnt->classes[d], my_classes);
        if (my_marks) atomicAdd(&cnt->marks[d], my_marks);
    }
}

// Second-level queue: the classes that mark some s <= smax (a few per cent
// of the leaders once 2^d exceeds smax) wait per warp until 32 are queued,
// so their minimal-polynomial work also runs on full warps.  Every lane of
// the warp calls push together; want marks the lanes that enqueue.
struct ClassQueue {
    u64 j[64], first[64], n[64];
};
template <typename Work>
GF2E_DEV void class_push(ClassQueue &q, int &qn, bool want, u64 j, u64 first, u64 n,
                         Work &&work) {
    const int lane = threadIdx.x & 31;
    const unsigned b = __ballot_sync(0xffffffffu, want);
    if (want) {
        const int pos = qn + __popc(b & ((1u << lane) - 1u));
        q.j[pos] = j;
        q.first[pos] = first;
        q.n[pos] = n;
    }
    qn += __popc(b);
    __syncwarp();
    if (qn >= 32) {
        const int pos = qn - 32 + lane;
        const u64 jj = q.j[pos], ff = q.first[pos], nn = q.n[pos];
        __syncwarp();
        qn -= 32;
        work(jj, ff, nn, true);
    }
}
template <typename Work>
GF2E_DEV void class_flush(ClassQueue &q, int qn, Work &&work) {
    const int lane = threadIdx.x & 31;
    const bool v = lane < qn;
    work(v ? q.j[lane] : 0, v ? q.first[lane] : 0, v ? q.n[lane] : 1, v);
}

__global__ void __launch_bounds__(256)
k_classes(const u32 *__restrict__ A, const u32 *__restrict__ L, const DegreeArgs a,
          unsigned long long *__restrict__ best, Prog *__restrict__ strip, Prog *__restrict__ heavy,
          Counters *__restrict__ cnt) {
    __shared__ u64 wq_all[8][64];
    __shared__ ClassQueue cq_all[8];
    const int d = a.d;
    const u64 M = a.M;
    unsigned long long my_classes = 0, my_marks = 0;
    ClassQueue &cq = cq_all[threadIdx.x >> 5];
    int cqn = 0;
    // minimal polynomial of beta = x^j (first linear dependency among
    // beta^0..beta^d over GF(2)) and the marks of its progression
    auto mark = [&](u64 j, u64 first, u64 n, bool valid) {
        if (!valid) return;
        const u64 count = (a.smax - first) / n + 1;
        u32 prow[DMAX + 1], ptag[DMAX + 1];
        int pbit[DMAX + 1];
        int np = 0;
        u32 mask = 0;
        u64 idx = 0;
        for (int k = 0; k <= d; k++) {
            u32 row = A[idx], tag = 1u << k;
            for (int p = 0; p < np; p++)
                if ((row >> pbit[p]) & 1) { row ^= prow[p]; tag ^= ptag[p]; }
            if (row == 0) { mask = tag; break; }
            pbit[np] = 31 - __clz(row);
            prow[np] = row;
            ptag[np] = tag;
            np++;
            idx += j;
            if (idx >= M) idx -= M;
        }
        if (!((mask >> d) & 1) || !(mask & 1)) {        // cannot happen
            atomicAdd(&cnt->bad, 1ull);
            return;
        }
        const unsigned long long key = ((u64)d << 48) | mask;
        my_marks += count;
        if (n < a.strip) {
            unsigned long long slot = atomicAdd(&cnt->nstrip, 1ull);
            if (slot < a.caps.strip) {
                strip[slot] = Prog{first, n, key};
            } else {
                atomicAdd(&cnt->spilled, 1ull);
                mark_inline(first, n, a.smax, key, best);
            }
        } else if (count <= INLINE) {
            mark_inline(first, n, a.smax, key, best);
        } else {
            unsigned long long slot = atomicAdd(&cnt->nheavy, 1ull);
            if (slot < a.caps.heavy) {
                heavy[slot] = Prog{first, n, key};
            } else {
                atomicAdd(&cnt->spilled, 1ull);
                mark_inline(first, n, a.smax, key, best);
            }
        }
    };
    for_each_leader(M, d, wq_all[threadIdx.x >> 5], [&](u64 j, bool valid) {
        bool ok = valid;
        for (int k = 0; k < a.nsub && ok; k++)
            if (j % a.subq[k] == 0) ok = false;
        u64 first = 0, n = 1;
        if (ok) {
            my_classes++;
            const u64 u = mod_mersenne(j * a.rmod, d, M);
            if (u == 0) ok = false;
            else ok = progression(j, L[A[u] ^ 1u], d, M, first, n) && first <= a.smax;
        }
        class_push(cq, cqn, ok, j, first, n, mark);
    });
    class_flush(cq, cqn, mark);
    add_stats(my_classes, my_marks, d, cnt);
}

// heavy progressions: block-strided over records, threads over marks
__global__ void k_heavy(const Prog *__restrict__ heavy, const Counters *__restrict__ cnt,
                        u64 smax, unsigned long long *__restrict__ best, u64 hcap) {
    u64 nh = cnt->nheavy;
    if (nh > hcap) nh = hcap;
    for (u64 rec = blockIdx.x; rec < nh; rec += gridDim.x) {
        Prog p = heavy[rec];
        for (u64 s = p.s0 + (u64)threadIdx.x * p.n; s <= smax; s += (u64)blockDim.x * p.n)
            atomicMin(&best[s], (unsigned long long)p.key);
    }
}

// short-period progressions, one STRIP-wide slice of best[] per CTA
__global__ void __launch_bounds__(512)
k_strip(const Prog *__restrict__ strip, const Counters *__restrict__ cnt, u64 smax,
        unsigned long long *__restrict__ best, const u64 STRIP, u64 scap) {
    extern __shared__ unsigned long long sb[];
    u64 ns = cnt->nstrip;
    if (ns > scap) ns = scap;
    const u64 nstrips = (smax + 1 + STRIP - 1) / STRIP;
    for (u64 sid = blockIdx.x; sid < nstrips; sid += gridDim.x) {
        const u64 lo = sid * STRIP;
        const u64 hi = (lo + STRIP - 1 < smax) ? lo + STRIP - 1 : smax;   // inclusive
        for (u64 i = threadIdx.x; i < STRIP; i += blockDim.x) sb[i] = ~0ull;
        __syncthreads();
        // warps take progressions, lanes take marks
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
        for (u64 pi = warp; pi < ns; pi += nwarps) {
            Prog p = strip[pi];
            if (p.s0 > hi) continue;
            u64 s = p.s0;
            if (s < lo) s += ((lo - s + p.n - 1) / p.n) * p.n;
            for (s += (u64)lane * p.n; s <= hi; s += 32 * p.n) atomicMin(&sb[s - lo], p.key);
        }
        __syncthreads();
        for (u64 i = threadIdx.x; i <= hi - lo; i += blockDim.x) {
            unsigned long long v = sb[i];
            if (v != ~0ull) {
                unsigned long long cur = best[lo + i];
                if (v < cur) best[lo + i] = v;
            }
        }
        __syncthreads();
    }
}

__global__ void k_fill(unsigned long long *p, u64 n, unsigned long long v) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (u64)gridDim.x * blockDim.x)
        p[i] = v;
}

// ---- wide field GF(2^d), 32 <= d <= 40: elements in 64 bits, modulus
// x^d + qlow with qlow of low degree e (2 e <= d), given by its terms
struct WideField {
    int d;
    int nt;                   // terms of qlow (bit positions, < d)
    int t[12];
    u64 M, qlow;
};

// t (hi:lo, below 2^(2d-1)) mod the modulus: two folds of the bits >= d by qlow
GF2E_DEV u64 wf_reduce(u64 lo, u64 hi, const WideField &F) {
    const int d = F.d;
    const u64 mask = F.M;                                // 2^d - 1
    u64 h = (lo >> d) | (hi << (64 - d));                // bits >= d, below 2^(d-1)
    u64 t = lo & mask;
    u64 f = 0;
#pragma unroll 4
    for (int i = 0; i < F.nt; i++) f ^= h << F.t[i];     // < 2^(d-1+e)
    t ^= f & mask;
    h = f >> d;                                          // below 2^(e-1)
    f = 0;
#pragma unroll 4
    for (int i = 0; i < F.nt; i++) f ^= h << F.t[i];     // < 2^(2e-1) <= 2^d
    return t ^ f;
}
GF2E_DEV u64 wf_mulx(u64 a, const WideField &F) {
    const u64 top = (a >> (F.d - 1)) & 1;
    return ((a << 1) & F.M) ^ (F.qlow & (0ull - top));
}
GF2E_DEV u64 wf_sqr(u64 a, const WideField &F) {
    return wf_reduce(spread32((u32)a), spread32((u32)(a >> 32)), F);
}
GF2E_DEV u64 wf_mul(u64 a, u64 b, const WideField &F) {
    const u32 a0 = (u32)a, a1 = (u32)(a >> 32), b0 = (u32)b, b1 = (u32)(b >> 32);
    const u64 lo = clmul32(a0, b0), hi = clmul32(a1, b1);
    const u64 mid = clmul32(a0 ^ a1, b0 ^ b1) ^ lo ^ hi;
    return wf_reduce(lo ^ (mid << 32), hi ^ (mid >> 32), F);
}
// x^e, e < 2^d: left to right, squaring then multiplying by x
GF2E_DEV u64 wf_powx(u64 e, const WideField &F) {
    if (!e) return 1;
    u64 r = 1;
    for (int bit = 63 - __clzll(e); bit >= 0; bit--) {
        r = wf_sqr(r, F);
        if ((e >> bit) & 1) r = wf_mulx(r, F);
    }
    return r;
}
// a * b mod M = 2^d - 1
GF2E_DEV u64 mulmod_mersenne(u64 a, u64 b, int d, u64 M) {
    unsigned __int128 p = (unsigned __int128)a * b;
    while (p > M) p = (p & M) + (p >> d);
    return p == M ? 0 : (u64)p;
}

// log-table slice: L[v - lo] = i for the values v = x^i in [lo, lo + len)
template <typename E>
__global__ void k_wide_slice(E *__restrict__ L, const WideField F, u64 lo, u64 len) {
    const u64 nchunk = (F.M + 63) >> 6;
    for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t < nchunk;
         t += (u64)gridDim.x * blockDim.x) {
        const u64 i0 = t << 6;
        u64 v = wf_powx(i0, F);
        const int ne = (int)min((u64)64, F.M - i0);
        for (int e = 0; e < ne; e++) {
            if (v - lo < len) L[v - lo] = (E)(i0 + e);
            v = wf_mulx(v, F);
        }
    }
}

struct WideArgs {
    WideField F;
    u64 rmod, smax, lo, len;
    int nsub, first_slice;
    u64 subq[6];
    ListCaps caps;
};

// a class of leader j whose progression (first, period n) reaches s <= smax:
// its minimal polynomial and the marks
GF2E_DEV void wide_mark(u64 j, u64 first, u64 n, const WideArgs &a,
                        unsigned long long *__restrict__ best, Prog *__restrict__ heavy,
                        Counters *__restrict__ cnt, unsigned long long &my_marks) {
    const int d = a.F.d;
    const u64 count = (a.smax - first) / n + 1;
    // minimal polynomial of beta = x^j: first linear dependency among
    // beta^0..beta^d over GF(2)
    const u64 beta = wf_powx(j, a.F);
    u64 prow[DMAX_WIDE + 1], ptag[DMAX_WIDE + 1];
    int pbit[DMAX_WIDE + 1];
    int np = 0;
    u64 mask = 0, pw = 1;
    for (int k = 0; k <= d; k++) {
        u64 row = pw, tag = 1ull << k;
        for (int p = 0; p < np; p++)
            if ((row >> pbit[p]) & 1) { row ^= prow[p]; tag ^= ptag[p]; }
        if (row == 0) { mask = tag; break; }
        pbit[np] = 63 - __clzll(row);
        prow[np] = row;
        ptag[np] = tag;
        np++;
        pw = wf_mul(pw, beta, a.F);
    }
    if (!((mask >> d) & 1) || !(mask & 1)) {        // cannot happen
        atomicAdd(&cnt->bad, 1ull);
        return;
    }
    const unsigned long long key = ((u64)d << 48) | mask;
    my_marks += count;
    if (count <= INLINE) {
        mark_inline(first, n, a.smax, key, best);
    } else {
        unsigned long long slot = atomicAdd(&cnt->nheavy, 1ull);
        if (slot < a.caps.heavy) {
            heavy[slot] = Prog{first, n, key};
        } else {
            atomicAdd(&cnt->spilled, 1ull);
            mark_inline(first, n, a.smax, key, best);
        }
    }
}


// one slice without a leader list: every leader recomputes x^(j r) + 1 and
// looks it up when it falls in this slice
template <typename E>
__global__ void __launch_bounds__(256)
k_wide_classes(const E *__restrict__ L, const WideArgs a, unsigned long long *__restrict__ best,
               Prog *__restrict__ heavy, Counters *__restrict__ cnt) {
    __shared__ u64 wq_all[8][64];
    __shared__ ClassQueue cq_all[8];
    const int d = a.F.d;
    const u64 M = a.F.M;
    unsigned long long my_classes = 0, my_marks = 0;
    ClassQueue &cq = cq_all[threadIdx.x >> 5];
    int cqn = 0;
    auto mark = [&](u64 j, u64 first, u64 n, bool valid) {
        if (valid) wide_mark(j, first, n, a, best, heavy, cnt, my_marks);
    };
    for_each_leader(M, d, wq_all[threadIdx.x >> 5], [&](u64 j, bool valid) {
        bool ok = valid;
        for (int k = 0; k < a.nsub && ok; k++)
            if (j % a.subq[k] == 0) ok = false;
        u64 w = 0, first = 0, n = 1;
        if (ok) {
            if (a.first_slice) my_classes++;
            const u64 u = mulmod_mersenne(j, a.rmod, d, M);
            if (u == 0) ok = false;
            else w = wf_powx(u, a.F) ^ 1ull;             // x^(j r) + 1
            ok = ok && w - a.lo < a.len;                  // else another slice's lookup
        }
        if (ok) ok = progression(j, (u64)L[w - a.lo], d, M, first, n) && first <= a.smax;
        class_push(cq, cqn, ok, j, first, n, mark);
    });
    class_flush(cq, cqn, mark);
    add_stats(my_classes, my_marks, d, cnt);
}

// once per degree: the leader list (j, x^(j r) + 1) of every class
__global__ void __launch_bounds__(256)
k_wide_leaders(const WideArgs a, ulonglong2 *__restrict__ list, u64 cap,
               Counters *__restrict__ cnt) {
    __shared__ u64 wq_all[8][64];
    const int d = a.F.d;
    const u64 M = a.F.M;
    const int lane = threadIdx.x & 31;
    unsigned long long my_classes = 0;
    for_each_leader(M, d, wq_all[threadIdx.x >> 5], [&](u64 j, bool valid) {
        bool keep = valid;
        for (int k = 0; k < a.nsub && keep; k++)
            if (j % a.subq[k] == 0) keep = false;
        u64 w = 0;
        if (keep) {
            my_classes++;
            const u64 u = mulmod_mersenne(j, a.rmod, d, M);
            if (u == 0) keep = false;
            else w = wf_powx(u, a.F) ^ 1ull;
        }
        const unsigned b = __ballot_sync(0xffffffffu, keep);
        if (!b) return;
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(&cnt->nlist, (unsigned long long)__popc(b));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (keep) {
            const u64 idx = base + __popc(b & ((1u << lane) - 1u));
            if (idx < cap) list[idx] = make_ulonglong2(j, w);
            else atomicAdd(&cnt->overflow, 1ull);
        }
    });
    add_stats(my_classes, 0, d, cnt);
}

// one slice with the leader list: the entries whose lookup lies in it
template <typename E>
__global__ void __launch_bounds__(256)
k_wide_match(const E *__restrict__ L, const ulonglong2 *__restrict__ list, u64 cap,
             const WideArgs a, unsigned long long *__restrict__ best, Prog *__restrict__ heavy,
             Counters *__restrict__ cnt) {
    __shared__ u64 wq_all[8][64];
    __shared__ ClassQueue cq_all[8];
    const u64 nl = min((u64)cnt->nlist, cap);
    const int d = a.F.d;
    const u64 M = a.F.M;
    unsigned long long my_marks = 0;
    ClassQueue &cq = cq_all[threadIdx.x >> 5];
    int cqn = 0;
    auto mark = [&](u64 j, u64 first, u64 n, bool valid) {
        if (valid) wide_mark(j, first, n, a, best, heavy, cnt, my_marks);
    };
    for_each_selected(
        0, nl, wq_all[threadIdx.x >> 5], [&](u64 i) { return list[i].y - a.lo < a.len; },
        [&](u64 i, bool valid) {
            u64 j = 0, first = 0, n = 1;
            bool ok = valid;
            if (ok) {
                const ulonglong2 e = list[i];
                j = e.x;
                ok = progression(j, (u64)L[e.y - a.lo], d, M, first, n) && first <= a.smax;
            }
            class_push(cq, cqn, ok, j, first, n, mark);
        });
    class_flush(cq, cqn, mark);
    add_stats(0, my_marks, a.F.d, cnt);
}

// ---- host-side field setup (gf2_field_setup.h:14-58 restated)
u32 h_mul(u32 a, u32 b, u64 q, int d) {
    u64 t = 0, x = a;
    while (b) { if (b & 1) t ^= x; x <<= 1; b >>= 1; }
    for (int bit = 2 * d - 2; bit >= d; bit--)
        if ((t >> bit) & 1) t ^= q << (bit - d);
    return (u32)t;
}
u32 h_pow(u32 base, u64 e, u64 q, int d) {
    u32 r = 1;
    while (e) { if (e & 1) r = h_mul(r, base, q, d); base = h_mul(base, base, q, d); e >>= 1; }
    return r;
}
int h_prime_factors(u64 m, u64 *out) {
    int n = 0;
    for (u64 p = 2; p * p <= m; p += (p == 2 ? 1 : 2))
        if (m % p == 0) { out[n++] = p; while (m % p == 0) m /= p; }
    if (m > 1) out[n++] = m;
    return n;
}
bool h_irreducible(u64 q, int d) {
    u32 chain[40];
    u32 t = 2;
    chain[0] = t;
    for (int i = 1; i <= d; i++) { t = h_mul(t, t, q, d); chain[i] = t; }
    if (chain[d] != 2) return false;
    u64 ps[16];
    int np = h_prime_factors((u64)d, ps);
    for (int i = 0; i < np; i++)
        if (chain[d / ps[i]] == 2) return false;
    return true;
}
u64 h_primitive(int d) {
    u64 M = ((u64)1 << d) - 1, ps[64];
    int np = h_prime_factors(M, ps);
    for (u64 q = ((u64)1 << d) | 1; q < ((u64)2 << d); q += 2) {
        if (!h_irreducible(q, d)) continue;
        bool prim = true;
        for (int i = 0; i < np && prim; i++)
            if (h_pow(2, M / ps[i], q, d) == 1) prim = false;
        if (prim) return q;
    }
    return 0;
}
// 64-bit elements for 33 <= d <= 40 (gf2_wide_setup.h:44-53 restated)
u64 hw_mul(u64 a, u64 b, u64 q, int d) {
    unsigned __int128 t = 0, x = a;
    while (b) { if (b & 1) t ^= x; x <<= 1; b >>= 1; }
    for (int bit = 2 * d - 2; bit >= d; bit--)
        if ((t >> bit) & 1) t ^= (unsigned __int128)q << (bit - d);
    return (u64)t;
}
u64 hw_pow(u64 base, u64 e, u64 q, int d) {
    u64 r = 1;
    while (e) { if (e & 1) r = hw_mul(r, base, q, d); base = hw_mul(base, base, q, d); e >>= 1; }
    return r;
}
bool hw_irreducible(u64 q, int d) {
    u64 chain[DMAX_WIDE + 1];
    u64 t = 2;
    chain[0] = t;
    for (int i = 1; i <= d; i++) { t = hw_mul(t, t, q, d); chain[i] = t; }
    if (chain[d] != 2) return false;
    u64 ps[16];
    int np = h_prime_factors((u64)d, ps);
    for (int i = 0; i < np; i++)
        if (chain[d / ps[i]] == 2) return false;
    return true;
}
u64 hw_primitive(int d) {
    u64 M = ((u64)1 << d) - 1, ps[64];
    int np = h_prime_factors(M, ps);
    for (u64 q = ((u64)1 << d) | 1; q < ((u64)2 << d); q += 2) {
        if (!hw_irreducible(q, d)) continue;
        bool prim = true;
        for (int i = 0; i < np && prim; i++)
            if (hw_pow(2, M / ps[i], q, d) == 1) prim = false;
        if (prim) return q;
    }
    return 0;
}
u64 cached_primitive(int d) {
    static std::mutex mu;
    static u64 cache[DMAX_WIDE + 1] = {0};
    std::lock_guard<std::mutex> lk(mu);
    if (!cache[d]) cache[d] = d <= 32 ? h_primitive(d) : hw_primitive(d);
    return cache[d];
}

// the wide field of degree d on its primitive polynomial; false if the low
// part of the modulus is too dense or too high for the two-fold reduction
bool wide_field(int d, WideField &F) {
    const u64 q = cached_primitive(d);
    if (!q) return false;
    const u64 qlow = q ^ ((u64)1 << d);
    F.d = d;
    F.M = ((u64)1 << d) - 1;
    F.qlow = qlow;
    F.nt = 0;
    int e = 0;
    for (int b = 0; b < d; b++)
        if ((qlow >> b) & 1) {
            if (F.nt == 12) return false;
            F.t[F.nt++] = b;
            e = b;
        }
    return 2 * e <= d;
}
u64 h_gcd(u64 a, u64 b) { while (b) { u64 t = a % b; a = b; b = t; } return a; }

}  // namespace

extern "C" {

uint64_t gf2e_primitive_poly(int d) {
    if (d < 2 || d > DMAX_WIDE) return 0;
    return cached_primitive(d);
}

int gf2e_sieve_workspace_size(int dmax, size_t *bytes) {
    if (dmax < 2 || dmax > DMAX_WIDE || !bytes)
        return gf2e::invalid("dmax must be in 2..%d", DMAX_WIDE);
    *bytes = layout().off_region + region_want(2, dmax);
    return GF2E_OK;
}

int gf2e_sieve_fill(uint64_t *best_dev, uint64_t smax, void *stream) {
    if (!best_dev) return gf2e::invalid("null best");
    k_fill<<<gf2e::grid_for(smax + 1, 256), 256, 0, (cudaStream_t)stream>>>(
        (unsigned long long *)best_dev, smax + 1, ~0ull);
    GF2E_CHECK_LAUNCH("k_fill");
    return GF2E_OK;
}

int gf2e_sieve_run(uint64_t r, int dmin, int dmax, uint64_t smax, uint64_t *best_dev,
                   void *workspace, size_t ws_bytes, void *stream) {
    if (dmin < 2 || dmax > DMAX_WIDE || dmin > dmax)
        return gf2e::invalid("degrees must satisfy 2 <= dmin <= dmax <= %d", DMAX_WIDE);
    if (!best_dev || !workspace || smax < 1 || r < 3)
        return gf2e::invalid("gf2e_sieve_run: bad arguments");
    const Layout lay = layout();
    const size_t need = lay.off_region + region_min(dmin, dmax);
    if (ws_bytes < need) return gf2e::invalid("sieve workspace %zu < %zu bytes", ws_bytes, need);
    const size_t region = ws_bytes - lay.off_region;
    // host-side checks and setup for every degree before any launch
    const int strip_log = gf2e::tune_current().sieve_strip_log;
    const u64 strip_w = (u64)1 << strip_log;
    std::vector<DegreeArgs> args;
    struct WidePlan {
        WideArgs a;
        bool list;                        // leader list at the region start
        size_t slice_off;                 // log-table slice offset in the region
        u64 list_cap;
    };
    std::vector<WidePlan> wargs;          // one per (wide degree, slice)
    const int wfrom = wide_from();
    const ListCaps caps = list_caps();
    for (int d = dmin; d <= dmax; d++) {
        const u64 M = ((u64)1 << d) - 1, rmod = r % M;
        if (h_gcd(rmod ? rmod : M, M) != 1) {
            gf2e::set_error("d=%d: gcd(r, 2^d-1) != 1; unsupported r", d);
            return GF2E_ERR_UNSUPPORTED_R;
        }
        u64 ps[16], subq[6];
        const int np = h_prime_factors((u64)d, ps);
        for (int i = 0; i < np; i++) subq[i] = M / (((u64)1 << (d / ps[i])) - 1);
        if (d < wfrom) {
            DegreeArgs a;
            memset(&a, 0, sizeof a);
            a.d = d;
            a.M = M;
            a.q = (u32)cached_primitive(d);
            a.rmod = rmod;
            a.smax = smax;
            a.strip = strip_w;
            a.caps = caps;
            a.nsub = np;
            for (int i = 0; i < np; i++) a.subq[i] = subq[i];
            args.push_back(a);
            continue;
        }
        WideArgs w;
        memset(&w, 0, sizeof w);
        if (!wide_field(d, w.F)) {
            gf2e::set_error("d=%d: primitive polynomial unsuitable for the wide field", d);
            return GF2E_ERR_INTERNAL;
        }
        w.rmod = rmod;
        w.smax = smax;
        w.caps = caps;
        w.nsub = np;
        for (int i = 0; i < np; i++) w.subq[i] = subq[i];
        // the leader list first in the region when it fits beside a slice of
        // at least 256 MB, then log-table slices: as few as the rest allows
        const size_t lb = leader_list_bytes(d);
        const bool use_list = leader_list_wanted(d) && region >= lb + ((size_t)1 << 28);
        const size_t slice_off = use_list ? lb : 0;
        const u64 values = (u64)1 << d, cap = (u64)((region - slice_off) / wide_entry_bytes(d));
        const u64 nslice = (values + cap - 1) / cap, len = (values + nslice - 1) / nslice;
        for (u64 b = 0; b < nslice; b++) {
            w.lo = b * len;
            w.len = std::min(len, values - w.lo);
            w.first_slice = b == 0;
            wargs.push_back(WidePlan{w, use_list, slice_off, use_list ? irreducible_count(d) : 0});
        }
    }
    {   // k_strip may take up to 2^STRIP_LOG_MAX entries of shared memory
        // set once per device; two threads racing here both set the same value
        static std::atomic<bool> attr_done[64];
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev >= 0 && dev < 64 && !attr_done[dev].load(std::memory_order_acquire)) {
            cudaError_t e = cudaFuncSetAttribute(k_strip, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)(sizeof(u64) << STRIP_LOG_MAX));
            if (e != cudaSuccess) return gf2e::cuda_status(e, "k_strip smem attribute");
            attr_done[dev].store(true, std::memory_order_release);
        }
    }
    cudaStream_t st = (cudaStream_t)stream;
    char *ws = (char *)workspace;
    Prog *strip = (Prog *)(ws + lay.off_strip);
    Prog *heavy = (Prog *)(ws + lay.off_heavy);
    Counters *cnt = (Counters *)(ws + lay.off_cnt);
    char *reg = ws + lay.off_region;
    cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(Counters), st);
    if (e != cudaSuccess) return gf2e::cuda_status(e, "sieve counters");
    unsigned long long *best = (unsigned long long *)best_dev;
    if (!args.empty()) {
        u32 *A = (u32 *)reg;
        u32 *L = (u32 *)(reg + dense_table_bytes(std::min(dmax, wfrom - 1)));
        for (const DegreeArgs &a : args) {
            u64 nchunk = (a.M + 31) >> 5;
            k_tables<<<gf2e::grid_for(nchunk, 256, 16), 256, 0, st>>>(A, L, a.d, a.q, a.M);
            GF2E_CHECK_LAUNCH("k_tables");
            k_classes<<<gf2e::grid_for(a.M, 256, 16), 256, 0, st>>>(A, L, a, best, strip, heavy,
                                                                    cnt);
            GF2E_CHECK_LAUNCH("k_classes");
        }
    }
    for (const WidePlan &P : wargs) {
        const WideArgs &w = P.a;
        const u64 nchunk = (w.F.M + 63) >> 6;
        const int gsl = gf2e::grid_for(nchunk, 256, 16), gcl = gf2e::grid_for(w.F.M, 256, 16);
        ulonglong2 *list = (ulonglong2 *)reg;
        char *slice = reg + P.slice_off;
        if (P.list && w.first_slice) {
            e = cudaMemsetAsync(&cnt->nlist, 0, sizeof(cnt->nlist), st);
            if (e != cudaSuccess) return gf2e::cuda_status(e, "sieve leader list");
            k_wide_leaders<<<gcl, 256, 0, st>>>(w, list, P.list_cap, cnt);
            GF2E_CHECK_LAUNCH("k_wide_leaders");
        }
        if (w.F.d <= 32) {
            k_wide_slice<u32><<<gsl, 256, 0, st>>>((u32 *)slice, w.F, w.lo, w.len);
            GF2E_CHECK_LAUNCH("k_wide_slice");
            if (P.list) {
                const u64 nl = P.list_cap;
                k_wide_match<u32><<<gf2e::grid_for(nl, 256, 16), 256, 0, st>>>(
                    (const u32 *)slice, list, P.list_cap, w, best, heavy, cnt);
            } else {
                k_wide_classes<u32><<<gcl, 256, 0, st>>>((const u32 *)slice, w, best, heavy, cnt);
            }
        } else {
            k_wide_slice<u64><<<gsl, 256, 0, st>>>((u64 *)slice, w.F, w.lo, w.len);
            GF2E_CHECK_LAUNCH("k_wide_slice");
            if (P.list) {
                const u64 nl = P.list_cap;
                k_wide_match<u64><<<gf2e::grid_for(nl, 256, 16), 256, 0, st>>>(
                    (const u64 *)slice, list, P.list_cap, w, best, heavy, cnt);
            } else {
                k_wide_classes<u64><<<gcl, 256, 0, st>>>((const u64 *)slice, w, best, heavy, cnt);
            }
        }
        GF2E_CHECK_LAUNCH("k_wide_classes");
    }
    k_heavy<<<gf2e::sm_count() * 16, 256, 0, st>>>(heavy, cnt, smax, best, caps.heavy);
    GF2E_CHECK_LAUNCH("k_heavy");
    u64 nstrips = (smax + strip_w) / strip_w;
    k_strip<<<gf2e::grid_for(nstrips * 512, 512, 2), 512, strip_w * sizeof(u64), st>>>(
        strip, cnt, smax, best, strip_w, caps.strip);
    GF2E_CHECK_LAUNCH("k_strip");
    // status: overflow / internal failures (one small read, synchronizes)
    unsigned long long flags[4];
    e = cudaMemcpyAsync(flags, cnt, sizeof flags, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return gf2e::cuda_status(e, "sieve status");
    if (flags[2]) {
        gf2e::set_error("sieve leader list overflow (%llu)", flags[2]);
        return GF2E_ERR_OVERFLOW;
    }
    if (flags[3]) {
        gf2e::set_error("minimal polynomial consistency failure (%llu classes)", flags[3]);
        return GF2E_ERR_INTERNAL;
    }
    return GF2E_OK;
}

int gf2e_sieve_stats(const void *workspace, int dmax, uint64_t *classes_host,
                     uint64_t *marks_host, void *stream) {
    if (!workspace || dmax < 2 || dmax > DMAX_WIDE)
        return gf2e::invalid("gf2e_sieve_stats: bad arguments");
    const Layout lay = layout();
    Counters c;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemcpyAsync(&c, (const char *)workspace + lay.off_cnt, sizeof c,
                                    cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return gf2e::cuda_status(e, "sieve stats");
    for (int d = 0; d <= dmax; d++) {
        if (classes_host) classes_host[d] = c.classes[d];
        if (marks_host) marks_host[d] = c.marks[d];
    }
    return GF2E_OK;
}

}  // extern "C"
