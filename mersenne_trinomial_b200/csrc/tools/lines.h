// lines.h -- the lines of a text file exactly as a loop of
// fgets(buf, 512, f) would see them (a line longer than 511 bytes arrives
// as several pieces), parsed by several threads and handed on in file
// order.  Host C++, no CUDA.
//
// The file is read in blocks of 64 MB, each cut at line starts into one
// piece per thread.  Every thread turns its piece into records with
// `parse`, and `apply` then sees the records of all pieces in file order,
// so anything order-dependent (first occurrences, messages) is decided as
// in the one-thread loop.
#pragma once

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace lines {

constexpr size_t kFgetsBytes = 511;          // fgets(buf, 512, f) returns at most 511

// parse(const char *p, size_t n, Rec &r) -> bool: one fgets chunk [p, p + n)
// (not NUL-terminated; it may hold NUL bytes, which end a C string there);
// true when the chunk yields a record.  apply(const Rec &) in file order.
template <class Rec, class Parse, class Apply>
bool for_each(FILE *f, Parse parse, Apply apply, int threads) {
    const int T = std::max(1, threads);
    constexpr size_t kBlock = (size_t)64 << 20;
    std::vector<char> rd(kBlock);
    std::string buf;
    bool eof = false;
    auto run_piece = [&](const char *b, const char *e, std::vector<Rec> &out) {
        out.clear();
        out.reserve((size_t)(e - b) / 16 + 1);
        Rec r;
        for (const char *p = b; p < e;) {
            const char *nl = (const char *)memchr(p, '\n', (size_t)(e - p));
            const char *le = nl ? nl + 1 : e;
            for (const char *q = p; q < le; q += kFgetsBytes) {
                const size_t n = std::min<size_t>(kFgetsBytes, (size_t)(le - q));
                if (parse(q, n, r)) out.push_back(r);
            }
            p = le;
        }
    };
    std::vector<std::vector<Rec>> outs(T);
    while (!eof) {
        const size_t n = fread(rd.data(), 1, rd.size(), f);
        if (n < rd.size()) {
            if (ferror(f)) return false;
            eof = true;
        }
        buf.append(rd.data(), n);
        size_t end = buf.size();
        if (!eof) {
            const size_t nl = buf.rfind('\n');
            if (nl == std::string::npos) continue;
            end = nl + 1;
        }
        std::vector<size_t> cut{0};
        for (int t = 1; t < T; t++) {
            const size_t at = end * (size_t)t / (size_t)T;
            if (at <= cut.back()) continue;
            const size_t nl = buf.find('\n', at - 1);
            if (nl == std::string::npos || nl + 1 >= end) break;
            if (nl + 1 > cut.back()) cut.push_back(nl + 1);
        }
        cut.push_back(end);
        const int np = (int)cut.size() - 1;
        std::vector<std::thread> pool;
        for (int i = 1; i < np; i++)
            pool.emplace_back([&, i] { run_piece(buf.data() + cut[i], buf.data() + cut[i + 1], outs[i]); });
        if (np > 0) run_piece(buf.data() + cut[0], buf.data() + cut[1], outs[0]);
        for (auto &th : pool) th.join();
        for (int i = 0; i < np; i++)
            for (const Rec &r : outs[i]) apply(r);
        buf.erase(0, end);
    }
    return true;
}

// [p, p + n) as a C string, the way a fgets buffer holding it reads
inline void c_string(const char *p, size_t n, char (&s)[kFgetsBytes + 1]) {
    memcpy(s, p, n);
    s[n] = '\0';
}

inline int default_threads() {
    const unsigned h = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min(h ? h : 1u, 32u));
}

}  // namespace lines
