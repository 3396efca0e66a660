// cert2bin -- certificate text to a found.bin image (the reference's
// cert2bin.c): one little-endian u64 per s = 1, 2, ... in order; "s u" and
// factors of degree above LIMIT become all ones, "s d p<hex>" becomes
// (d << 48) | mask with the mask exactly d + 1 bits long.
//
//   cert2bin <input_text_file> <output_binary_file> <LIMIT>      (LIMIT <= 47)
//
// Any format error names the line and exits 1, like the reference.
#include <cctype>
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

typedef uint64_t u64;

namespace {

[[noreturn]] void fail(u64 line, const char *what) {
    fprintf(stderr, "Error: %s at line %" PRIu64 "\n", what, line);
    exit(EXIT_FAILURE);
}

struct Reader {
    FILE *f;
    std::vector<char> buf = std::vector<char>(1 << 16);
    size_t pos = 0, len = 0;
    int get() {
        if (pos == len) {
            len = fread(buf.data(), 1, buf.size(), f);
            pos = 0;
            if (!len) return EOF;
        }
        return (unsigned char)buf[pos++];
    }
};

int hexval(int c) {
    if (c >= '0' && c <= '9') return c - '0';
    c = tolower(c);
    return (c >= 'a' && c <= 'f') ? c - 'a' + 10 : -1;
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
    Reader in{fopen(argv[1], "rb")};
    if (!in.f) { perror("Error opening input text file"); return EXIT_FAILURE; }
    FILE *out = fopen(argv[2], "wb");
    if (!out) { perror("Error opening output binary file"); fclose(in.f); return EXIT_FAILURE; }
    std::vector<u64> block;
    block.reserve(8192);
    auto emit = [&](u64 v) {
        block.push_back(v);
        if (block.size() == 8192) { fwrite(block.data(), 8, block.size(), out); block.clear(); }
    };
    auto skip_line = [&](int c) { while (c != '\n' && c != EOF) c = in.get(); };
    for (u64 want = 1;; want++) {
        int c;
        do c = in.get(); while (c == ' ' || c == '\t' || c == '\n' || c == '\r');
        if (c == EOF) break;
        if (!isdigit(c)) fail(want, "Expected line number");
        u64 s = 0;
        for (; isdigit(c); c = in.get()) s = s * 10 + (u64)(c - '0');
        if (s != want) {
            fprintf(stderr, "Error: Expected line number %" PRIu64 ", got %" PRIu64 "\n", want, s);
            exit(EXIT_FAILURE);
        }
        while (c == ' ' || c == '\t') c = in.get();
        if (c == 'u') { emit(~0ull); skip_line(c); continue; }
        if (!isdigit(c)) fail(want, "Expected 'u' or integer 'd'");
        u64 d = 0;
        for (; isdigit(c); c = in.get()) d = d * 10 + (u64)(c - '0');
        while (c == ' ' || c == '\t') c = in.get();
        if (c != 'p') fail(want, "Expected 'p'");
        if (d > (u64)limit) { emit(~0ull); skip_line(c); continue; }
        u64 mask = 0;
        for (c = in.get(); c != '\n' && c != '\r' && c != ' ' && c != EOF; c = in.get()) {
            const int h = hexval(c);
            if (h < 0) fail(want, "Invalid hex character");
            mask = (mask << 4) | (u64)h;
        }
        if ((mask >> d) != 1) fail(want, "Hex value bit size is not exactly d+1");
        emit((d << 48) | mask);                  // anything after the mask starts the next record
    }
    if (!block.empty()) fwrite(block.data(), 8, block.size(), out);
    fclose(in.f);
    fclose(out);
    return EXIT_SUCCESS;
}
