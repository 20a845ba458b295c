// bpc_train.cu -- LUT training: symbol statistics gathered on the GPU and
// written as LUT text files in the reference's format.
//
// The reference ships trained probability tables (LUTs/) but no trainer.  A
// LUT entry is the 7-bit probability, out of 128, that the symbol coded with
// it is 0 (Arithmetic_encoder, BPC_PaCo.cu:261-295: the interval part of
// symbol 0 is (Size * P) >> 7).  Training counts, for every entry of the
// layout load_LUTs builds (main_example.cu:219-448) with 15 planes, how many
// symbols the coder codes with it and how many of them are 1, then writes
// P = round(128 * zeros / symbols) clamped to 1..127 (64, p = 1/2, for entries
// no symbol used).
//
// Files.  One record per line, "<level> <subband> <plane> : p0 .. pN-1", the
// (level, subband) groups in layout order (level 0 HL, LH, HH, level 1, ...,
// the LL band as level `levels` subband 0).  Each group lists planes 0..t,
// where t is one past its highest plane with data (at most 14), and plane t is
// all 64: load_LUTs overwrites a group's last listed plane from its second
// entry on with 64 when the next group starts (main_example.cu:292-299), so the
// shipped tables end every group that way and these do too.  (A group with data
// in plane 14 therefore keeps only the first entry of its plane-14 record.)
// The last group (LL) always lists planes 0..14, as in the shipped tables:
// load_LUTs sizes its sections by the largest plane the files list
// (:231-278), and the coder's addressing assumes 15.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <string>

#include "../../include/bpc_paco.h"
#include "bpc_core.cuh"
#include "bpc_kernels.h"

namespace {
constexpr int kPlanes = 15;
}

extern "C" int bpc_lut_stats(const int *d_coeffs, int X, int Y, int passes, int levels, int cb_size,
                             unsigned long long *d_stats, void *stream) {
    if (!d_coeffs || !d_stats || (passes != 2 && passes != 3) || levels < 1 || levels > 16 ||
        (cb_size != 64 && cb_size != 32) || X <= 0 || Y <= 0 || X % cb_size || Y % cb_size ||
        (long long)X * Y > (1LL << 31) - 1 || !bpc::aligned_to(d_coeffs, bpc::kEncInAlign))
        return BPC_ERR_ARG;
    const int n = bpc_lut_entries(passes, levels, kPlanes);
    const bpc::LutOffsets o = bpc::lut_offsets(levels, passes, n);
    bpc::Params p;
    p.in = d_coeffs;
    p.out = nullptr;
    p.lut = nullptr;
    p.lut_n = n;
    p.tab_n = o.tab_n;
    p.X = X;
    p.Y = Y;
    p.levels = levels;
    p.ncbx = X / cb_size;
    p.ncb = (X / cb_size) * (Y / cb_size);
    p.a_sig = o.a_sig;
    p.a_sign = o.a_sign;
    p.cp_off = o.cp_off;
    p.status = nullptr;
    p.counts = nullptr;
    p.offsets = nullptr;
    p.cb_begin = 0;
    p.cb_end = p.ncb;
    const cudaError_t e = bpc::launch_stats(passes, cb_size, p, d_stats, (cudaStream_t)stream);
    if (e != cudaSuccess) {
        std::fprintf(stderr, "bpc: LUT statistics kernel: %s\n", cudaGetErrorString(e));
        return BPC_ERR_CUDA;
    }
    return BPC_OK;
}

extern "C" int bpc_lut_write(const char *folder, const unsigned long long *stats, int passes, int levels) {
    if (!folder || !stats || (passes != 2 && passes != 3) || levels < 1 || levels > 16) return BPC_ERR_ARG;
    struct Section {
        const char *name;
        int nctx;
    };
    const Section secs[5] = {{"ref.txt", 1}, {"sig.txt", 9}, {"sign.txt", 4}, {"cp_sig.txt", 9}, {"cp_sign.txt", 4}};
    const int ngroups = 3 * levels + 1;
    long base = 0;
    for (int si = 0; si < (passes == 3 ? 5 : 3); ++si) {
        const Section &sec = secs[si];
        const std::string path = std::string(folder) + sec.name;
        FILE *f = std::fopen(path.c_str(), "w");
        if (!f) {
            std::fprintf(stderr, "bpc: cannot create %s\n", path.c_str());
            return BPC_ERR_FILE;
        }
        for (int gi = 0; gi < ngroups; ++gi) {
            const int level = gi / 3, sb = gi % 3;
            const long g0 = base + (long)gi * kPlanes * sec.nctx;
            int last = -1;  // highest plane with a coded symbol
            for (int b = 0; b < kPlanes; ++b)
                for (int k = 0; k < sec.nctx; ++k)
                    if (stats[2 * (g0 + (long)b * sec.nctx + k)]) last = b;
            // the LL group lists all 15 planes: load_LUTs sizes its sections by
            // the largest plane in the files, and the coder addresses 15
            int t = last + 1 < kPlanes ? last + 1 : kPlanes - 1;
            if (gi == ngroups - 1) t = kPlanes - 1;
            for (int b = 0; b <= t; ++b) {
                std::fprintf(f, "%d %d %d :", level, sb, b);
                for (int k = 0; k < sec.nctx; ++k) {
                    const long idx = g0 + (long)b * sec.nctx + k;
                    const unsigned long long n = stats[2 * idx], ones = stats[2 * idx + 1];
                    int P = 64;
                    if (n && b <= last) {
                        const double q = 128.0 * (double)(n - ones) / (double)n;
                        P = (int)std::lround(q);
                        P = P < 1 ? 1 : (P > 127 ? 127 : P);
                    }
                    std::fprintf(f, " %d", P);
                }
                std::fprintf(f, " \n");
            }
        }
        const bool ok = std::fclose(f) == 0;
        if (!ok) return BPC_ERR_FILE;
        base += 3L * kPlanes * sec.nctx * levels + (long)kPlanes * sec.nctx;
    }
    return BPC_OK;
}
