// bpc_lut.cpp -- host LUT loader with the semantics of load_LUTs
// (PabloEnfedaque/CUDA_BPC-PaCo source/main_example.cu:219-448).
//
// File format, one record per line:  "<level> <subband> <bitplane> : p0 .. pN-1"
// with N = 1 (ref.txt), 9 (sig.txt, cp_sig.txt), 4 (sign.txt, cp_sign.txt).
// Layout rules kept from the reference (the kernel's addressing depends on them):
//   * max_bitplane = 1 + the largest bitplane column of ref/sig/sign (:231-264);
//   * sections ref | sig | sign [| cp_sig | cp_sign], each
//     (3 * mb * N * levels + mb * N) ints (:266-278);
//   * a record whose bitplane does not exceed the previous one starts a new
//     (level, subband) group: the previous group's span from entry prev*N + 1
//     to its end is set to 64 and the cursor moves by mb*N (:292-299);
//   * the level/subband columns are not read.
// Defined where the reference is not: entries nothing writes are 0 (the
// reference leaves malloc garbage), writes past the array are dropped (the
// reference overruns its heap buffer when `levels` is smaller than the files'
// group count), and a malformed record is an error (the reference loops).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "bpc_lut.h"

namespace bpc {

namespace {

struct Record {
    int bitplane;
    int v[9];
};

// Parses every record of one file.  Returns 0, or a negative BPC_ERR_* code.
int parse_file(const std::string &path, int nvals, std::vector<Record> &out) {
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return kErrFile;
    std::string text;
    char buf[1 << 14];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, got);
    std::fclose(f);
    const char *s = text.c_str();
    const char *end = s + text.size();
    auto skip = [&]() {
        while (s < end && (*s == ' ' || *s == '\t' || *s == '\r' || *s == '\n')) s++;
    };
    auto read_int = [&](long &v) -> bool {
        skip();
        if (s >= end) return false;
        char *e = nullptr;
        v = std::strtol(s, &e, 10);
        if (e == s) return false;
        s = e;
        return true;
    };
    for (;;) {
        skip();
        if (s >= end) break;
        long lvl, sb, bp, x;
        if (!read_int(lvl) || !read_int(sb) || !read_int(bp)) return kErrParse;
        skip();
        if (s >= end || *s != ':') return kErrParse;
        s++;
        Record r;
        r.bitplane = (int)bp;
        for (int k = 0; k < nvals; k++) {
            if (!read_int(x)) return kErrParse;
            r.v[k] = (int)x;
        }
        out.push_back(r);
    }
    return 0;
}

void place_section(const std::vector<Record> &recs, int nctx, int mb, long base, int *lut, long total) {
    long cursor = base;
    int prev = -1;
    auto put = [&](long idx, int v) {
        if (idx >= 0 && idx < total) lut[idx] = v;
    };
    for (const Record &r : recs) {
        if (r.bitplane <= prev) {
            const long first = cursor + (long)prev * nctx + 1;
            const long last = cursor + (long)mb * nctx;  // inclusive, as the reference's fill loop
            for (long k = first; k <= last; k++) put(k, 64);
            cursor += (long)mb * nctx;
        }
        prev = r.bitplane;
        for (int k = 0; k < nctx; k++) put(cursor + (long)r.bitplane * nctx + k, r.v[k]);
    }
}

}  // namespace

long lut_section_size(int mb, int nctx, int levels) { return 3L * mb * nctx * levels + (long)mb * nctx; }

long lut_entries(int passes, int levels, int mb) {
    const long r = lut_section_size(mb, 1, levels), g = lut_section_size(mb, 9, levels),
               n = lut_section_size(mb, 4, levels);
    return passes == 3 ? r + 2 * g + 2 * n : r + g + n;
}

int load_luts_host(const char *folder, int passes, int levels, std::vector<int> &lut) {
    if (!folder || (passes != 2 && passes != 3) || levels < 1 || levels > 16) return kErrArg;
    static const char *names[5] = {"ref.txt", "sig.txt", "sign.txt", "cp_sig.txt", "cp_sign.txt"};
    static const int nctx[5] = {1, 9, 4, 9, 4};
    const int nfiles = passes == 3 ? 5 : 3;
    std::vector<Record> recs[5];
    for (int f = 0; f < nfiles; f++) {
        const int rc = parse_file(std::string(folder) + names[f], nctx[f], recs[f]);
        if (rc) return rc;
    }
    int mb = -1;
    for (int f = 0; f < 3; f++)
        for (const Record &r : recs[f]) mb = r.bitplane > mb ? r.bitplane : mb;
    mb += 1;
    if (mb <= 0 || mb > 64) return kErrParse;
    const long total = lut_entries(passes, levels, mb);
    lut.assign((size_t)total, 0);
    const long r = lut_section_size(mb, 1, levels), g = lut_section_size(mb, 9, levels),
               n = lut_section_size(mb, 4, levels);
    const long base[5] = {0, r, r + g, r + g + n, r + 2 * g + n};
    for (int f = 0; f < nfiles; f++) place_section(recs[f], nctx[f], mb, base[f], lut.data(), total);
    return 0;
}

}  // namespace bpc
