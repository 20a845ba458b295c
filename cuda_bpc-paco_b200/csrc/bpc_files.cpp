// bpc_files.cpp -- per-codeblock stream files, the on-disk form of the slot
// stream read by load_CStream (PabloEnfedaque/CUDA_BPC-PaCo
// source/main_example.cu:51-68) in the file numbering of load_Data (:71-179).
//
// File k of a folder prefix is "<prefix><k>.bin": the cb*cb words of one
// codeblock's slot, each as a 16-bit big-endian value (the MSB word, the
// codewords, then the fill).  Codeblocks are numbered as load_Data walks them:
// the LL band first, then for level = levels..1 the HL, LH and HH bands, each
// band in raster order of cb x cb blocks; file k lands in the slot of the
// codeblock at that position of the raster.  Reading mirrors load_CStream: a
// word is (first byte << 8) | second byte, and a byte past the end of the file
// makes the word -1 (fgetc's EOF in both halves of the OR).  Unlike the
// reference a missing file is an error instead of a crash.
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/bpc_paco.h"

namespace {

struct Pos {
    int x0, y0;
};

// codeblock origins in load_Data order (:82-179)
std::vector<Pos> file_order(int X, int Y, int levels, int cb) {
    std::vector<Pos> out;
    auto band = [&](int ox, int oy, int w, int h) {
        for (int j = 0; j < h; j += cb)
            for (int i = 0; i < w; i += cb) out.push_back({ox + i, oy + j});
    };
    band(0, 0, X >> levels, Y >> levels);
    for (int lv = levels; lv > 0; --lv) {
        const int w = X >> lv, h = Y >> lv;
        band(w, 0, w, h);
        band(0, h, w, h);
        band(w, h, w, h);
    }
    return out;
}

bool valid(const char *folder, int X, int Y, int levels, int cb) {
    return folder && X > 0 && Y > 0 && (cb == 64 || cb == 32) && X % cb == 0 && Y % cb == 0 && levels >= 0 &&
           levels <= 16;
}

std::string name(const char *folder, int k) { return std::string(folder) + std::to_string(k) + ".bin"; }

size_t slot_of(const Pos &q, int X, int cb) {
    return ((size_t)(q.y0 / cb) * (size_t)(X / cb) + (size_t)(q.x0 / cb)) * (size_t)cb * (size_t)cb;
}

}  // namespace

extern "C" int bpc_load_cstreams(const char *folder, int *stream, int X, int Y, int levels, int cb_size) {
    if (!stream || !valid(folder, X, Y, levels, cb_size)) return BPC_ERR_ARG;
    const std::vector<Pos> order = file_order(X, Y, levels, cb_size);
    const size_t n = (size_t)cb_size * (size_t)cb_size;
    std::vector<unsigned char> buf(2 * n);
    for (size_t k = 0; k < order.size(); ++k) {
        FILE *f = std::fopen(name(folder, (int)k).c_str(), "rb");
        if (!f) {
            std::fprintf(stderr, "bpc: cannot open %s\n", name(folder, (int)k).c_str());
            return BPC_ERR_FILE;
        }
        const size_t got = std::fread(buf.data(), 1, buf.size(), f);
        std::fclose(f);
        int *slot = stream + slot_of(order[k], X, cb_size);
        for (size_t i = 0; i < n; ++i)
            slot[i] = 2 * i + 1 < got ? ((int)buf[2 * i] << 8) | (int)buf[2 * i + 1] : -1;
    }
    return BPC_OK;
}

extern "C" int bpc_save_cstreams(const char *folder, const int *stream, int X, int Y, int levels, int cb_size) {
    if (!stream || !valid(folder, X, Y, levels, cb_size)) return BPC_ERR_ARG;
    const std::vector<Pos> order = file_order(X, Y, levels, cb_size);
    const size_t n = (size_t)cb_size * (size_t)cb_size;
    std::vector<unsigned char> buf(2 * n);
    for (size_t k = 0; k < order.size(); ++k) {
        const int *slot = stream + slot_of(order[k], X, cb_size);
        for (size_t i = 0; i < n; ++i) {
            buf[2 * i] = (unsigned char)((slot[i] >> 8) & 0xFF);
            buf[2 * i + 1] = (unsigned char)(slot[i] & 0xFF);
        }
        FILE *f = std::fopen(name(folder, (int)k).c_str(), "wb");
        if (!f) {
            std::fprintf(stderr, "bpc: cannot create %s\n", name(folder, (int)k).c_str());
            return BPC_ERR_FILE;
        }
        const size_t put = std::fwrite(buf.data(), 1, buf.size(), f);
        if (std::fclose(f) != 0 || put != buf.size()) return BPC_ERR_FILE;
    }
    return BPC_OK;
}

extern "C" int bpc_cstream_files(int X, int Y, int levels, int cb_size) {
    if (!valid("", X, Y, levels, cb_size)) return BPC_ERR_ARG;
    return (int)file_order(X, Y, levels, cb_size).size();
}
