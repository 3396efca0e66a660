// certfmt.h -- text output of sieve results (host C++, no CUDA).
//
// The line formats are the reference's (coarse_sieve.cu:1510-1558,
// bin2cert.c): a certificate line "s d p<hex>" (decimal s, decimal degree,
// lowercase hex mask without leading zeros), a survivor line "s", and
// bin2cert's "s u" for an all-ones record.  The bytes are those of
// printf("%" PRIu64 " %u p%" PRIx64 "\n", ...); the conversions are written
// out here, and ranges of s are formatted by several threads into per-chunk
// buffers that are then written in order.  At r = 136279841 (68 M values
// of s, 63 M certificate lines) formatting with one printf per line takes
// seconds, against milliseconds for the sieve itself.
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <string>
#include <thread>
#include <vector>

namespace certfmt {

typedef uint64_t u64;

constexpr u64 kNone = ~0ull;                 // all-ones key: no factor yet
constexpr u64 kMaskBits = 0xFFFFFFFFFFFFull; // low 48 bits: the mask

inline char *put_dec(char *p, u64 v) {
    char t[20];
    int n = 0;
    do {
        t[n++] = (char)('0' + v % 10);
        v /= 10;
    } while (v);
    while (n) *p++ = t[--n];
    return p;
}

inline char *put_hex(char *p, u64 v) {
    static const char dig[] = "0123456789abcdef";
    const int nd = v ? (67 - __builtin_clzll(v)) / 4 : 1;
    for (int i = nd - 1; i >= 0; i--) *p++ = dig[(v >> (4 * i)) & 15];
    return p;
}

// "s d p<hex>\n" for key v = (d << 48) | mask
inline char *put_cert(char *p, u64 s, u64 v) {
    p = put_dec(p, s);
    *p++ = ' ';
    p = put_dec(p, v >> 48);
    *p++ = ' ';
    *p++ = 'p';
    p = put_hex(p, v & kMaskBits);
    *p++ = '\n';
    return p;
}

enum class Lines {
    Cert,        // coarse_sieve .found.cert: every s with a key (not all ones, not 0)
    Survivors,   // coarse_sieve .survivors.txt: every s with no key
    Bin2Cert,    // bin2cert: "s u" for no key, else the certificate line
};

// Lines for keys[i], i in [i0, i1), of s = s_of_0 + i; returns lines made.
inline u64 format_range(const u64 *keys, u64 i0, u64 i1, u64 s_of_0, Lines kind,
                        std::string &out) {
    out.clear();
    out.reserve((size_t)(i1 - i0) * (kind == Lines::Survivors ? 10 : 24));
    char line[64];
    u64 n = 0;
    for (u64 i = i0; i < i1; i++) {
        const u64 v = keys[i], s = s_of_0 + i;
        char *p = line;
        switch (kind) {
        case Lines::Cert:
            if (v == kNone || v == 0) continue;
            p = put_cert(p, s, v);
            break;
        case Lines::Survivors:
            if (v != kNone) continue;
            p = put_dec(p, s);
            *p++ = '\n';
            break;
        case Lines::Bin2Cert:
            if (v == kNone) {
                p = put_dec(p, s);
                *p++ = ' ';
                *p++ = 'u';
                *p++ = '\n';
            } else {
                p = put_cert(p, s, v);
            }
            break;
        }
        out.append(line, (size_t)(p - line));
        n++;
    }
    return n;
}

inline int default_threads() {
    const unsigned h = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min(h ? h : 1u, 32u));
}

// Write the lines of keys[0..n) (s = s_of_0 + i) to f, formatted by
// `threads` threads in rounds of at most 2^22 keys.  Returns the number of
// lines, or -1 when a write fails.
inline long long write_lines(FILE *f, const u64 *keys, u64 n, u64 s_of_0, Lines kind,
                             int threads = default_threads()) {
    constexpr u64 kRound = (u64)1 << 22;
    const int T = std::max(1, threads);
    std::vector<std::string> buf(T);
    std::vector<u64> cnt(T);
    long long total = 0;
    for (u64 r0 = 0; r0 < n; r0 += kRound) {
        const u64 r1 = std::min(n, r0 + kRound), per = (r1 - r0 + T - 1) / T;
        std::vector<std::thread> pool;
        for (int t = 0; t < T; t++) {
            const u64 a = std::min(r1, r0 + t * per), b = std::min(r1, a + per);
            if (t == 0)
                continue;
            pool.emplace_back([&, t, a, b] { cnt[t] = format_range(keys, a, b, s_of_0, kind, buf[t]); });
        }
        cnt[0] = format_range(keys, r0, std::min(r1, r0 + per), s_of_0, kind, buf[0]);
        for (auto &th : pool) th.join();
        for (int t = 0; t < T; t++) {
            if (!buf[t].empty() && fwrite(buf[t].data(), 1, buf[t].size(), f) != buf[t].size())
                return -1;
            total += (long long)cnt[t];
        }
    }
    return total;
}

}  // namespace certfmt
