// cert2bin -- certificate text to a found.bin image (the reference's
// cert2bin.c): one little-endian u64 per s = 1, 2, ... in order; "s u" and
// factors of degree above LIMIT become all ones, "s d p<hex>" becomes
// (d << 48) | mask with the mask exactly d + 1 bits long.
//
//   cert2bin <input_text_file> <output_binary_file> <LIMIT>      (LIMIT <= 47)
//
// Any format error names the line and exits 1, like the reference.
//
// The text is read in blocks and each block is cut at line starts into
// pieces parsed by several threads.  A line start is always between records
// (every record ends within its line), so a piece parses exactly as it
// would in one pass, except that it cannot know which s its first record
// must carry: each piece records its first s, its record count and its
// first error, and the pieces are then checked in file order against the
// running record number, so the first error reported, its message and its
// line number are those of the one-pass reading.
#include <algorithm>
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

typedef uint64_t u64;

namespace {

enum Err { OK = 0, NO_LINE_NUMBER, LINE_ORDER, NO_DEGREE, NO_P, BAD_HEX, BAD_BITS };

struct Piece {
    std::vector<u64> vals;
    u64 first_s = 0, nrec = 0;   // records begun (the erring one included)
    bool has_first = false;
    Err err = OK;
    u64 err_rec = 0, got = 0;    // record index in the piece; the s found (LINE_ORDER)
};

int hexval(unsigned char c) {
    if (c >= '0' && c <= '9') return c - '0';
    if (c >= 'a' && c <= 'f') return c - 'a' + 10;
    if (c >= 'A' && c <= 'F') return c - 'A' + 10;
    return -1;
}
bool digit(int c) { return c >= '0' && c <= '9'; }

// Parse [b, e) (starting at a line start) into p.  `limit`: degrees above it
// become all ones.
void parse_piece(const char *b, const char *e, u64 limit, Piece &p) {
    const char *q = b;
    auto get = [&]() -> int { return q < e ? (unsigned char)*q++ : EOF; };
    auto skip_line = [&](int c) { while (c != '\n' && c != EOF) c = get(); };
    auto fail = [&](Err k) { p.err = k; p.err_rec = p.nrec - 1; };
    p.vals.reserve((size_t)(e - b) / 16 + 1);
    for (;;) {
        int c;
        do c = get(); while (c == ' ' || c == '\t' || c == '\n' || c == '\r');
        if (c == EOF) return;
        p.nrec++;
        if (!digit(c)) return fail(NO_LINE_NUMBER);
        u64 s = 0;
        for (; digit(c); c = get()) s = s * 10 + (u64)(c - '0');
        if (!p.has_first) {
            p.has_first = true;
            p.first_s = s;
        } else if (s != p.first_s + (p.nrec - 1)) {
            p.got = s;
            return fail(LINE_ORDER);
        }
        while (c == ' ' || c == '\t') c = get();
        if (c == 'u') {
            p.vals.push_back(~0ull);
            skip_line(c);
            continue;
        }
        if (!digit(c)) return fail(NO_DEGREE);
        u64 d = 0;
        for (; digit(c); c = get()) d = d * 10 + (u64)(c - '0');
        while (c == ' ' || c == '\t') c = get();
        if (c != 'p') return fail(NO_P);
        if (d > limit) {
            p.vals.push_back(~0ull);
            skip_line(c);
            continue;
        }
        u64 mask = 0;
        for (c = get(); c != '\n' && c != '\r' && c != ' ' && c != EOF; c = get()) {
            const int h = hexval((unsigned char)c);
            if (h < 0) return fail(BAD_HEX);
            mask = (mask << 4) | (u64)h;
        }
        if ((mask >> d) != 1) return fail(BAD_BITS);
        p.vals.push_back((d << 48) | mask);      // anything after the mask starts the next record
    }
}

[[noreturn]] void report(Err k, u64 line, u64 got) {
    static const char *what[] = {"", "Expected line number", "", "Expected 'u' or integer 'd'",
                                 "Expected 'p'", "Invalid hex character",
                                 "Hex value bit size is not exactly d+1"};
    if (k == LINE_ORDER)
        fprintf(stderr, "Error: Expected line number %" PRIu64 ", got %" PRIu64 "\n", line, got);
    else
        fprintf(stderr, "Error: %s at line %" PRIu64 "\n", what[k], line);
    exit(EXIT_FAILURE);
}

}  // namespace

int main(int argc, char **argv) {
    if (argc != 4) {
        fprintf(stderr, "Usage: %s <input_text_file> <output_binary_file> <LIMIT>\n", argv[0]);
        return EXIT_FAILURE;
    }
    const long limit = strtol(argv[3], nullptr, 10);
    if (limit > 47) {
        fprintf(stderr, "Error: LIMIT cannot be greater than 47 (would overflow 48-bit field).\n");
        return EXIT_FAILURE;
    }
    FILE *in = fopen(argv[1], "rb");
    if (!in) { perror("Error opening input text file"); return EXIT_FAILURE; }
    FILE *out = fopen(argv[2], "wb");
    if (!out) { perror("Error opening output binary file"); fclose(in); return EXIT_FAILURE; }
    const u64 lim = (u64)limit;   // compared as unsigned, as the reference's d > limit is
    const unsigned hw = std::thread::hardware_concurrency();
    const int T = (int)std::max(1u, std::min(hw ? hw : 1u, 32u));
    constexpr size_t kBlock = (size_t)64 << 20;
    std::string buf;                               // carried partial line + the new block
    std::vector<char> rd(kBlock);
    u64 want = 1;                                  // the next record's s
    bool eof = false;
    while (!eof) {
        const size_t n = fread(rd.data(), 1, rd.size(), in);
        if (n < rd.size()) eof = true;
        buf.append(rd.data(), n);
        // complete lines only, unless this is the end of the input
        size_t end = buf.size();
        if (!eof) {
            const size_t nl = buf.rfind('\n');
            if (nl == std::string::npos) continue;
            end = nl + 1;
        }
        // pieces cut at line starts
        std::vector<size_t> cut{0};
        for (int t = 1; t < T; t++) {
            size_t at = end * (size_t)t / (size_t)T;
            if (at <= cut.back()) continue;
            const size_t nl = buf.find('\n', at - 1);
            if (nl == std::string::npos || nl + 1 >= end) break;
            if (nl + 1 > cut.back()) cut.push_back(nl + 1);
        }
        cut.push_back(end);
        const int np = (int)cut.size() - 1;
        std::vector<Piece> ps(np);
        std::vector<std::thread> pool;
        for (int i = 1; i < np; i++)
            pool.emplace_back([&, i] { parse_piece(buf.data() + cut[i], buf.data() + cut[i + 1], lim, ps[i]); });
        if (np > 0) parse_piece(buf.data() + cut[0], buf.data() + cut[1], lim, ps[0]);
        for (auto &th : pool) th.join();
        for (const Piece &p : ps) {
            if (p.has_first && p.first_s != want) report(LINE_ORDER, want, p.first_s);
            if (p.err != OK) report(p.err, want + p.err_rec, p.got);
            if (!p.vals.empty() && fwrite(p.vals.data(), 8, p.vals.size(), out) != p.vals.size()) {
                fprintf(stderr, "Error writing output binary file.\n");
                return EXIT_FAILURE;
            }
            want += p.nrec;
        }
        buf.erase(0, end);
    }
    fclose(in);
    if (fclose(out) != 0) { fprintf(stderr, "Error writing output binary file.\n"); return EXIT_FAILURE; }
    return EXIT_SUCCESS;
}
