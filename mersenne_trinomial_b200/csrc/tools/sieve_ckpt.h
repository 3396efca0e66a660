// sieve_ckpt.h -- checkpoint files of the coarse sieve (host C++, no CUDA).
//
// A checkpoint holds best[] (the packed key (d << 48) | mask per s, all ones
// for "no factor yet") and the point to resume from.  The file layout is the
// reference's version-2 checkpoint (coarse_sieve.cu:509-831), so a run
// stopped under either tool resumes under the other:
//
//   8 bytes   magic "GF2SVCK2"
//   6 x u32   version 2, degree d, next bucket, buckets of degree d,
//             baseline kind (0 none, 1 .found.bin image, 2 survivors list),
//             baseline path length
//   6 x u64   r, smax, depth, periodic interval in whole seconds,
//             FNV-1a hash of the baseline's keys s = 1..smax (0 without one),
//             number of delta entries
//   baseline path (no terminator)
//   payload   full image: smax u64 keys, s = 1..smax;
//             delta: (s, key) u64 pairs where best[] differs from the baseline
//
// Meaning: every degree below d is complete in best[], and of degree d the
// buckets [0, next) are.  This engine has no buckets (a wide degree runs its
// slices inside one library call); it writes degree boundaries as (d, 0, 0)
// and resumes a mid-degree file by running degree d whole, which is exact
// because best[] only ever takes minima.
//
// All values little-endian (the reference writes its structs raw on x86).
#pragma once

#include <cinttypes>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace sieve_ckpt {

typedef uint64_t u64;
typedef uint32_t u32;

static const char kMagic[8] = {'G', 'F', '2', 'S', 'V', 'C', 'K', '2'};
constexpr int kGenerationsTried = 8;   // path, path.1 .. path.7 on resume

// where a run stands: degrees < d done, buckets [0, next) of d done
struct Point {
    int d = 0, next = 0, nbuckets = 0;
};

// the --load / --load-survivors image a delta checkpoint is taken against
struct Baseline {
    int kind = 0;                      // 0 none, 1 found.bin, 2 survivors list
    std::string path;
    std::vector<u64> image;            // smax + 1 entries, index 0 unused
    u64 hash = 0;
    bool usable(u64 smax) const { return kind != 0 && image.size() == smax + 1; }
};

// FNV-1a over the keys as 64-bit units (offset basis and prime of FNV-1a 64)
inline u64 image_hash(const u64 *keys, u64 n) {
    u64 h = 0xcbf29ce484222325ull;
    for (u64 i = 0; i < n; i++) {
        h ^= keys[i];
        h *= 0x100000001b3ull;
    }
    return h;
}

// A .found.bin image: exactly smax LE u64 keys for s = 1..smax.
inline bool load_found(const char *path, u64 smax, std::vector<u64> &out, FILE *err = stderr) {
    FILE *f = fopen(path, "rb");
    if (!f) {
        if (err) fprintf(err, "%s: cannot open\n", path);
        return false;
    }
    fseek(f, 0, SEEK_END);
    long long bytes = ftell(f);
    fseek(f, 0, SEEK_SET);
    if (bytes != (long long)(smax * 8)) {
        if (err)
            fprintf(err, "%s: %lld bytes, smax=%" PRIu64 " needs %" PRIu64
                         " (smax must match the earlier run)\n",
                    path, bytes, smax, smax * 8);
        fclose(f);
        return false;
    }
    out.assign(smax + 1, ~0ull);
    const bool ok = fread(out.data() + 1, 8, smax, f) == smax;
    fclose(f);
    if (!ok && err) fprintf(err, "%s: short read\n", path);
    return ok;
}

// A survivors list (one s per line): listed s open (all ones), every other
// s gets 0, a key below any degree the run will sieve, so no mark lands
// there -- the sieve only compares keys, it never reads their masks.
inline bool load_survivors(const char *path, u64 smax, std::vector<u64> &out, u64 *listed = nullptr,
                           u64 *out_of_range = nullptr, FILE *err = stderr) {
    FILE *f = fopen(path, "r");
    if (!f) {
        if (err) fprintf(err, "%s: cannot open\n", path);
        return false;
    }
    out.assign(smax + 1, 0);
    u64 n = 0, oor = 0;
    char line[128];
    while (fgets(line, sizeof line, f)) {
        char *end = nullptr;
        const u64 s = strtoull(line, &end, 10);
        if (end == line) continue;
        if (s < 1 || s > smax) {
            oor++;
            continue;
        }
        out[s] = ~0ull;
        n++;
    }
    fclose(f);
    if (listed) *listed = n;
    if (out_of_range) *out_of_range = oor;
    return true;
}

inline bool load_baseline(Baseline &b, u64 smax, FILE *err = stderr) {
    if (b.kind == 1) return load_found(b.path.c_str(), smax, b.image, err);
    if (b.kind == 2) return load_survivors(b.path.c_str(), smax, b.image, nullptr, nullptr, err);
    return false;
}

// path.(keep-1) is dropped, path.i -> path.(i+1), path -> path.1
inline void rotate(const std::string &path, int keep) {
    if (keep <= 1) return;
    remove((path + "." + std::to_string(keep - 1)).c_str());
    for (int i = keep - 2; i >= 0; i--) {
        const std::string from = i == 0 ? path : path + "." + std::to_string(i);
        rename(from.c_str(), (path + "." + std::to_string(i + 1)).c_str());
    }
}

struct WriteInfo {
    bool delta = false;
    u64 entries = 0;                   // delta entries, or smax for a full image
    u64 bytes = 0;
};

// Write best[] at point `pt`: to path.tmp, then rotate the generations and
// rename, so an interrupted write never replaces a good file.  A delta
// against the baseline is written when it is smaller than the full image.
inline bool write(const std::string &path, int keep, u64 r, u64 smax, int depth, double period_s,
                  const Point &pt, const std::vector<u64> &best, const Baseline &base,
                  WriteInfo *info = nullptr, FILE *err = stderr) {
    if (best.size() != smax + 1) return false;
    std::vector<u64> pairs;
    bool delta = base.usable(smax);
    if (delta) {
        for (u64 s = 1; s <= smax && delta; s++) {
            if (best[s] == base.image[s]) continue;
            pairs.push_back(s);
            pairs.push_back(best[s]);
            if (pairs.size() * 8 >= smax * 8) delta = false;   // no smaller than full
        }
        if (!delta) pairs.clear();
    }
    const std::string tmp = path + ".tmp";
    FILE *f = fopen(tmp.c_str(), "wb");
    if (!f) {
        if (err) fprintf(err, "%s: cannot create\n", tmp.c_str());
        return false;
    }
    const u32 plen = delta ? (u32)base.path.size() : 0;
    const u32 h32[6] = {2u, (u32)pt.d, (u32)pt.next, (u32)pt.nbuckets, delta ? (u32)base.kind : 0u,
                        plen};
    const u64 nd = delta ? (u64)(pairs.size() / 2) : 0;
    const u64 h64[6] = {r, smax, (u64)depth, (u64)(period_s + 0.5), delta ? base.hash : 0ull, nd};
    bool ok = fwrite(kMagic, 1, 8, f) == 8 && fwrite(h32, 4, 6, f) == 6 && fwrite(h64, 8, 6, f) == 6;
    if (ok && plen) ok = fwrite(base.path.data(), 1, plen, f) == plen;
    if (ok) {
        if (delta)
            ok = pairs.empty() || fwrite(pairs.data(), 8, pairs.size(), f) == pairs.size();
        else
            ok = fwrite(best.data() + 1, 8, smax, f) == smax;
    }
    ok = (fflush(f) == 0) && ok;
    ok = (fclose(f) == 0) && ok;
    if (!ok) {
        if (err) fprintf(err, "checkpoint write failed (%s)\n", tmp.c_str());
        remove(tmp.c_str());
        return false;
    }
    rotate(path, keep);
    if (rename(tmp.c_str(), path.c_str()) != 0) {
        if (err) fprintf(err, "%s: rename failed\n", path.c_str());
        return false;
    }
    if (info) {
        info->delta = delta;
        info->entries = delta ? nd : smax;
        info->bytes = 8 + 24 + 48 + plen + (delta ? 16 * nd : 8 * smax);
    }
    return true;
}

// Read one checkpoint file for (r, smax).  A delta file reloads its
// baseline (which must hash as recorded) and applies the pairs; the
// baseline is handed back so later checkpoints of the resumed run can be
// deltas too.  A completed last degree (next >= nbuckets > 0) is
// normalised to the start of the next degree.
inline bool read_one(const std::string &path, u64 r, u64 smax, std::vector<u64> &best, Point &pt,
                     double &period_s, Baseline &base, FILE *err = stderr) {
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return false;
    auto fail = [&](const char *why) {
        if (err) fprintf(err, "%s: %s\n", path.c_str(), why);
        fclose(f);
        return false;
    };
    char magic[8];
    u32 h32[6];
    u64 h64[6];
    if (fread(magic, 1, 8, f) != 8 || memcmp(magic, kMagic, 8) != 0)
        return fail("not a version-2 sieve checkpoint");
    if (fread(h32, 4, 6, f) != 6 || fread(h64, 8, 6, f) != 6) return fail("truncated header");
    if (h64[0] != r || h64[1] != smax) {
        if (err)
            fprintf(err, "%s: written for r=%" PRIu64 " smax=%" PRIu64 ", this run has r=%" PRIu64
                         " smax=%" PRIu64 "\n",
                    path.c_str(), h64[0], h64[1], r, smax);
        fclose(f);
        return false;
    }
    const int kind = (int)h32[4];
    if (h32[5] > 4096) return fail("implausible baseline path length");
    std::string bpath(h32[5], '\0');
    if (h32[5] && fread(&bpath[0], 1, h32[5], f) != h32[5]) return fail("truncated baseline path");
    if (kind != 0) {
        Baseline b;
        b.kind = kind;
        b.path = bpath;
        if (kind != 1 && kind != 2) return fail("unknown baseline kind");
        if (!load_baseline(b, smax, err)) return fail("its baseline file cannot be read");
        b.hash = image_hash(b.image.data() + 1, smax);
        if (b.hash != h64[4]) return fail("its baseline file is not the one it was written against");
        best = b.image;
        for (u64 i = 0; i < h64[5]; i++) {
            u64 pr[2];
            if (fread(pr, 8, 2, f) != 2) return fail("truncated delta");
            if (pr[0] < 1 || pr[0] > smax) return fail("delta entry outside 1..smax");
            best[pr[0]] = pr[1];
        }
        base = std::move(b);
    } else {
        best.assign(smax + 1, ~0ull);
        if (fread(best.data() + 1, 8, smax, f) != smax) return fail("truncated image");
    }
    fclose(f);
    pt.d = (int)h32[1];
    pt.next = (int)h32[2];
    pt.nbuckets = (int)h32[3];
    if (pt.nbuckets > 0 && pt.next >= pt.nbuckets) {
        pt.d += 1;
        pt.next = pt.nbuckets = 0;
    }
    period_s = (double)h64[3];
    return true;
}

// Newest generation first, then path.1, path.2, ...: a damaged newest file
// falls back to the one before it.  `used` names the file that was read.
inline bool read(const std::string &path, u64 r, u64 smax, std::vector<u64> &best, Point &pt,
                 double &period_s, Baseline &base, std::string *used = nullptr,
                 FILE *err = stderr) {
    for (int i = 0; i < kGenerationsTried; i++) {
        const std::string g = i == 0 ? path : path + "." + std::to_string(i);
        FILE *probe = fopen(g.c_str(), "rb");
        if (!probe) {
            if (i == 0) continue;
            break;
        }
        fclose(probe);
        if (read_one(g, r, smax, best, pt, period_s, base, err)) {
            if (used) *used = g;
            return true;
        }
        if (err) fprintf(err, "checkpoint %s unusable; trying an older generation\n", g.c_str());
    }
    if (err) fprintf(err, "--resume %s: no usable checkpoint generation\n", path.c_str());
    return false;
}

}  // namespace sieve_ckpt
