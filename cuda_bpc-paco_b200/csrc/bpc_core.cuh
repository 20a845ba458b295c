// bpc_core.cuh -- BPC-PaCo codeblock coder, one warp per 64x64 codeblock
// (two 16-lane groups per warp for 32x32 codeblocks).
//
// Bitstream contract (PabloEnfedaque/CUDA_BPC-PaCo, source/BPC_PaCo.cu):
//   * lane l of a codeblock owns the 2-column stripe at columns 2l, 2l+1 and
//     runs its own fixed-probability arithmetic coder (:261-339);
//   * planes b = MSB..0, passes SPP, MRP [, CP] (3-pass: an extra CP at MSB,
//     :968-1090), rows 0..H-1, left column then right column (:633-962);
//   * within one step all lanes make their significance/refinement call, then
//     the lanes that became significant make their sign call; an exhausted lane
//     reserves the next codeword slot in ascending lane order (__ballot/__popc,
//     :268-279).  That reservation order IS the bitstream.
//
// Representation (new): instead of one 32-bit word per coefficient with flag
// bits (:1120), every lane keeps its state as 64-bit column masks (bit i =
// row i): significance S, refinement-eligible R, CP-pending C and sign N, plus
// copies of the two neighbour columns (lane-1's right column, lane+1's left
// column) that are kept current with one ballot per step that changes them.
// A context is a popcount of a 9-bit neighbourhood gathered from three 3-row
// windows; there are no per-coefficient shuffles.  Magnitudes are held as
// bitplanes (one 64-bit row mask per plane and column) in a per-thread array
// built with an in-register 32x32 bit transpose; the decoder collects decoded
// planes the same way and transposes them back at the end.  No shared memory
// is reserved per codeblock except the decoder's codeword ring, so a CTA of 4
// warps fits 7 times per SM.  The LUT sits in shared memory as bytes.
//
// The code is written against a small warp interface W (lane id, ballot, any,
// shuffles, syncwarp) so the same source runs as a CUDA kernel (bpc_kernels.cu).
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define BPC_FI __device__ __forceinline__
#else
#define BPC_FI inline
#endif

namespace bpc {

enum : int { ST_OVERFLOW = 1, ST_BAD_STREAM = 2, ST_INPUT_RANGE = 4, ST_LUT_RANGE = 8 };
enum : int { PK_SPP = 0, PK_MRP = 1, PK_CP = 2 };

// Sign-context table of Compute_Sign_Context (:178-211), indexed by
// (class(h) * 3 + class(v)), class = 0 for 0, 1 for > 0, 2 for < 0; 3 bits each.
constexpr uint32_t kSignTab = (0u << 0) | (2u << 3) | (3u << 6) | (4u << 9) | (6u << 12) | (0u << 15) |
                              (5u << 18) | (1u << 21) | (7u << 24);

struct Params {
    const int32_t *in;   // encode: raster coefficients; decode: slot stream
    int32_t *out;        // encode: slot stream; decode: raster coefficients
    const int32_t *lut;  // loader array (ints)
    int lut_n;           // its length
    int tab_n;           // shared byte table length (covers every index the coder forms)
    int X, Y, levels;
    int ncbx, ncb;       // codeblocks per row, total
    int a_sig, a_sign, cp_off;  // LUT section offsets as the reference kernel forms them
    int *status;         // OR of ST_* bits, may be null
    int *counts;         // per-codeblock codeword count, may be null
};

// LUT offsets the reference kernel uses (Initialize_LUT_pointers :228-250 with
// LUT_N_BITPLANES = 15, and the CP offset :988-989).
struct LutOffsets {
    int a_sig, a_sign, cp_off, tab_n;
};
inline LutOffsets lut_offsets(int levels, int passes, int lut_n) {
    LutOffsets o;
    const int ref_n = 3 * 15 * 1 * levels + 15 * 1;
    const int sig_n = 3 * 15 * 9 * levels + 15 * 9;
    const int sign_n = 3 * 15 * 4 * levels + 15 * 4;
    o.a_sig = ref_n;
    o.a_sign = ref_n + sig_n;
    o.cp_off = sig_n + sign_n;
    // largest index formed: LL group (levels*45) at plane 32 (all-zero block)
    const int gmax = levels * 45 + 32;
    int mx = gmax;  // refinement
    int s1 = o.a_sig + gmax * 9 + 8, s2 = o.a_sign + gmax * 4 + 3;
    if (passes == 3) {
        s1 += o.cp_off;
        s2 += o.cp_off;
    }
    mx = mx > s1 ? mx : s1;
    mx = mx > s2 ? mx : s2;
    int n = mx + 1;
    if (n < lut_n) n = lut_n;
    o.tab_n = (n + 15) & ~15;
    return o;
}

template <int CBS>
struct Geo {
    static constexpr int NL = CBS / 2;                   // lanes per codeblock
    static constexpr int NG = 32 / NL;                   // codeblocks per warp
    static constexpr int CAP = CBS * CBS;                // slot size in ints
    static constexpr int RING = CBS == 64 ? 512 : 256;   // decoder ring per codeblock
    static constexpr int CHUNK = RING / 2;               // refill size
    static constexpr int RING_WORDS = RING * NG;         // per warp
    static constexpr uint64_t ROWS = CBS == 64 ? ~0ull : 0xffffffffull;
};

BPC_FI uint32_t win3(uint64_t m, int i) {
    uint64_t t = i ? (m >> (i - 1)) : (m << 1);
    return (uint32_t)t & 7u;
}

BPC_FI int popc32(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return __popc(x);
#else
    return __builtin_popcount(x);
#endif
}
BPC_FI int ctz64(uint64_t x) {
#if defined(__CUDA_ARCH__)
    return __ffsll((long long)x) - 1;
#else
    return __builtin_ctzll(x);
#endif
}
BPC_FI int clz32(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return __clz(x);
#else
    return x ? __builtin_clz(x) : 32;
#endif
}

// In-register transpose of a 32x32 bit matrix, LSB first: afterwards bit r of
// a[c] is what bit c of a[r] was.  (Recursive block swap; 5 x 16 exchanges.)
BPC_FI void transpose32(uint32_t a[32]) {
    uint32_t m = 0x0000FFFFu;
#pragma unroll
    for (int j = 16; j; j >>= 1, m ^= m << j) {
#pragma unroll
        for (int k = 0; k < 32; k = (k + j + 1) & ~j) {
            const uint32_t t = ((a[k] >> j) ^ a[k + j]) & m;
            a[k + j] ^= t;
            a[k] ^= t << j;
        }
    }
}

struct Lane {
    uint64_t S[2], R[2], C[2], N[2];
    uint64_t XL, XR, XNL, XNR;
    uint32_t lower, size, resv, cw;
    uint32_t cnt;      // codewords reserved in this codeblock (group-uniform)
    uint32_t ring_hi;  // decoder: slot words [ring_hi - RING, ring_hi) are in the ring
    int has_resv;
    int status;
};

template <class W>
BPC_FI uint64_t warp_or64(W &w, uint64_t v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        uint32_t lo = w.shfl_xor((uint32_t)v, o), hi = w.shfl_xor((uint32_t)(v >> 32), o);
        v |= ((uint64_t)hi << 32) | lo;
    }
    return v;
}

template <class W>
BPC_FI uint64_t shfl_up64(W &w, uint64_t v) {
    uint32_t lo = w.shfl_up((uint32_t)v, 1), hi = w.shfl_up((uint32_t)(v >> 32), 1);
    return ((uint64_t)hi << 32) | lo;
}
template <class W>
BPC_FI uint64_t shfl_down64(W &w, uint64_t v) {
    uint32_t lo = w.shfl_down((uint32_t)v, 1), hi = w.shfl_down((uint32_t)(v >> 32), 1);
    return ((uint64_t)hi << 32) | lo;
}

template <int PASSES, int CBS, bool ENC, class W>
struct Coder {
    using G = Geo<CBS>;
    static constexpr int NH = CBS / 32;  // 32-row halves per column
    W &w;
    const Params &p;
    Lane s;
    uint32_t *ring;      // per codeblock (decoder)
    const uint8_t *tab;  // LUT bytes
    const int32_t *slot_in;
    int32_t *slot_out;
    int lane, gl, g, msb;
    int top;  // highest stored bitplane (-1: none)
    uint32_t gmask, ltmask;
    uint64_t B[2];  // encoder: magnitude bits of the current plane; decoder: decoded 1-bits
    int sig_base, sign_base;  // LUT byte indices of the current plane and pass
    // bitplanes, [plane][col0 rows 0-31, col0 rows 32-63, col1 rows 0-31, col1 rows 32-63]
    uint32_t planes[28][4];

    BPC_FI Coder(W &w_, const Params &p_, uint32_t *ring_all, const uint8_t *tab_) : w(w_), p(p_), tab(tab_) {
        lane = w.lane();
        gl = lane % G::NL;
        const int grp = lane / G::NL;
        gmask = G::NL == 32 ? 0xffffffffu : (0xffffu << (grp * 16));
        ltmask = (1u << lane) - 1u;
        ring = ring_all + grp * G::RING;
    }

    // ---------------------------------------------------------------- AC
    // Arithmetic_encoder :261-295
    BPC_FI void ac_enc(bool act, uint32_t sym, uint32_t P) {
        const bool need = act && s.size == 0;
        const uint32_t bal = w.ballot(need) & gmask;
        if (need) {
            s.resv = 1u + s.cnt + (uint32_t)popc32(bal & ltmask);
            s.has_resv = 1;
            s.lower = 0;
            s.size = 0xFFFFu;
        }
        s.cnt += (uint32_t)popc32(bal);
        if (act) {
            const uint32_t t = ((s.size * P) >> 7) + sym;
            if (sym) {
                s.size -= t;
                s.lower += t;
            } else {
                s.size = t;
            }
            if (s.size == 0) {
                if (s.resv < (uint32_t)G::CAP)
                    slot_out[s.resv] = (int32_t)s.lower;
                else
                    s.status |= ST_OVERFLOW;
            }
        }
    }

    // Arithmetic_decoder :297-339; the codeword is read when it is reserved
    BPC_FI uint32_t ac_dec(bool act, uint32_t P) {
        const bool need = act && s.size == 0;
        const uint32_t bal = w.ballot(need) & gmask;
        if (need) {
            const uint32_t idx = 1u + s.cnt + (uint32_t)popc32(bal & ltmask);
            if (idx < (uint32_t)G::CAP) {
                s.cw = ring[idx & (G::RING - 1)];
            } else {
                s.cw = 0xFFFFFFFFu;
                s.status |= ST_OVERFLOW;
            }
            s.lower = 0;
            s.size = 0xFFFFu;
        }
        s.cnt += (uint32_t)popc32(bal);
        uint32_t sym = 0;
        if (act) {
            const uint32_t t = ((s.size * P) >> 7) + 1u;
            const uint32_t thr = s.lower + t;
            if (s.cw >= thr) {
                s.size -= t;
                s.lower = thr;
                sym = 1;
            } else {
                s.size = t - 1u;
            }
        }
        return sym;
    }

    // decoder: make sure ring holds slot words [cnt+1, cnt+1+2*NL)
    BPC_FI void ring_load(uint32_t first, int nwords) {
        // group-cooperative, 16-byte loads; words past the slot read as -1
        const int per = nwords / G::NL;  // 8 or 16, multiple of 4
        for (int q = 0; q < per; q += 4) {
            const uint32_t k = first + (uint32_t)(gl * per + q);
            uint32_t v0, v1, v2, v3;
            if (k + 3 < (uint32_t)G::CAP) {
                w.load4(slot_in + k, v0, v1, v2, v3);
            } else {
                v0 = k + 0 < (uint32_t)G::CAP ? (uint32_t)slot_in[k + 0] : 0xFFFFFFFFu;
                v1 = k + 1 < (uint32_t)G::CAP ? (uint32_t)slot_in[k + 1] : 0xFFFFFFFFu;
                v2 = k + 2 < (uint32_t)G::CAP ? (uint32_t)slot_in[k + 2] : 0xFFFFFFFFu;
                v3 = k + 3 < (uint32_t)G::CAP ? (uint32_t)slot_in[k + 3] : 0xFFFFFFFFu;
            }
            const uint32_t r = k & (G::RING - 1);
            ring[r] = v0;
            ring[r + 1] = v1;
            ring[r + 2] = v2;
            ring[r + 3] = v3;
        }
    }
    BPC_FI void ring_ensure() {
        if (s.cnt + 1u + 2u * G::NL > s.ring_hi) {  // group-uniform
            w.syncmask(gmask);
            ring_load(s.ring_hi, G::CHUNK);
            s.ring_hi += G::CHUNK;
            w.syncmask(gmask);
        }
    }

    // Decoder reconstruction: the reference ORs a plane mask 3 << b into the
    // coefficient (:1038-1083); every bit it sets is later replaced by the
    // decoded bit, so the output holds exactly the decoded bits -- except for
    // MSB = 32, where 3 << 32 is 0 and the mask stays 0 until plane 0.
    BPC_FI bool keep_bit(int b) const { return msb != 32 || b == 0; }

    // Data bit the encoder codes at plane b: magnitude bit b for b <= 27; above
    // that the reference reads its flag bits (b+1 = 29 R, 30 C, 31 sigma, 32+
    // nothing), which for the coefficients each pass visits gives these
    // constants.  Planes >= 28 are only visited by all-zero codeblocks (MSB 32).
    template <int PK>
    BPC_FI uint32_t data_bit(int i, int c, int b) {
        if (b <= 27) return (uint32_t)(B[c] >> i) & 1u;
        if (PK == PK_CP) return b == 29 ? 1u : 0u;
        if (PK == PK_MRP) return (b == 28 || b == 30) ? 1u : 0u;
        return 0u;
    }

    // plane registers: encoder loads the magnitude bits, decoder clears
    BPC_FI void plane_begin(int b) {
        if (ENC) {
            if (b <= top) {
                const uint32_t *q = planes[b];
                B[0] = (uint64_t)q[0] | ((uint64_t)q[1] << 32);
                B[1] = (uint64_t)q[2] | ((uint64_t)q[3] << 32);
            } else {
                B[0] = B[1] = 0ull;
            }
        } else {
            B[0] = B[1] = 0ull;
        }
    }
    BPC_FI void plane_end(int b) {
        if (!ENC && b <= 27 && keep_bit(b)) {
            uint32_t *q = planes[b];
            q[0] = (uint32_t)B[0];
            q[1] = (uint32_t)(B[0] >> 32);
            q[2] = (uint32_t)B[1];
            q[3] = (uint32_t)(B[1] >> 32);
        }
    }

    // ------------------------------------------------------- context steps
    template <int PK, int c>
    BPC_FI void ctx_step(int i, int b, bool act) {
        const uint64_t bit = 1ull << i;
        const bool cand = act && (PK == PK_SPP ? !((s.S[c] >> i) & 1) : ((s.C[c] >> i) & 1));
        if (!w.any(cand)) return;
        if (!ENC) ring_ensure();
        const uint64_t Lm = c ? s.S[0] : s.XL, Mm = s.S[c], Rm = c ? s.XR : s.S[1];
        const uint32_t wl = win3(Lm, i), wm = win3(Mm, i), wr = win3(Rm, i);
        const uint32_t nbh = wl | ((wm & 5u) << 3) | (wr << 6);
        bool coded = cand;
        if (PK == PK_SPP && PASSES == 3) {
            if (cand && nbh == 0) {
                s.C[c] |= bit;  // SPP defers to CP (:450-452)
                coded = false;
            }
        }
        const int ctx = popc32(nbh);
        const uint32_t P = coded ? tab[sig_base + ctx] : 0u;
        uint32_t sym;
        if (ENC) {
            sym = coded ? data_bit<PK>(i, c, b) : 0u;
            ac_enc(coded, sym, P);
        } else {
            sym = ac_dec(coded, P);
        }
        if (PK == PK_CP && coded) s.C[c] &= ~bit;
        const bool ns = coded && sym && b <= 27;
        if (ns) {
            s.S[c] |= bit;
            if (PK == PK_CP) s.R[c] |= bit;
            if (!ENC) B[c] |= bit;
        }
        if (!w.any(ns)) return;
        // sign call (Compute_Sign_Context :214-226 over u, l, r, b)
        const uint64_t LN = c ? s.N[0] : s.XNL, MN = s.N[c], RN = c ? s.XNR : s.N[1];
        const int ls = (wl >> 1) & 1, rs = (wr >> 1) & 1, us = wm & 1, bs = (wm >> 2) & 1;
        const int ln = (int)((LN >> i) & 1), rn = (int)((RN >> i) & 1);
        const uint32_t wmn = win3(MN, i);
        const int un = wmn & 1, bn = (wmn >> 2) & 1;
        const int h = ls * (1 - 2 * ln) + rs * (1 - 2 * rn);
        const int v = us * (1 - 2 * un) + bs * (1 - 2 * bn);
        const int hc = h == 0 ? 0 : (h > 0 ? 1 : 2), vc = v == 0 ? 0 : (v > 0 ? 1 : 2);
        const int sctx = (int)((kSignTab >> (3 * (hc * 3 + vc))) & 7u);
        const uint32_t P2 = ns ? tab[sign_base + (sctx >> 1)] : 0u;
        uint32_t neg;
        if (ENC) {
            neg = (uint32_t)((s.N[c] >> i) & 1);
            ac_enc(ns, neg ^ (uint32_t)(sctx & 1), P2);
        } else {
            neg = ac_dec(ns, P2) ^ (uint32_t)(sctx & 1);
            if (ns && neg) s.N[c] |= bit;
        }
        // neighbour columns: lane l's column c at row i changed
        const uint32_t bsig = w.ballot(ns);
        const uint32_t bneg = ENC ? 0u : w.ballot(ns && neg);
        if (c == 0) {
            if (gl < G::NL - 1) {
                s.XR |= (uint64_t)((bsig >> (lane + 1)) & 1u) << i;
                if (!ENC) s.XNR |= (uint64_t)((bneg >> (lane + 1)) & 1u) << i;
            }
        } else {
            if (gl > 0) {
                s.XL |= (uint64_t)((bsig >> (lane - 1)) & 1u) << i;
                if (!ENC) s.XNL |= (uint64_t)((bneg >> (lane - 1)) & 1u) << i;
            }
        }
    }

    template <int PK>
    BPC_FI void ctx_pass(int b, bool act) {
        const int off = PK == PK_CP ? p.cp_off : 0;
        sig_base = off + p.a_sig + (g + b) * 9;
        sign_base = off + p.a_sign + (g + b) * 4;
        const uint64_t c0 = act ? (PK == PK_SPP ? ~s.S[0] : s.C[0]) : 0ull;
        const uint64_t c1 = act ? (PK == PK_SPP ? ~s.S[1] : s.C[1]) : 0ull;
        uint64_t U = warp_or64(w, (c0 | c1) & G::ROWS);
        while (U) {
            const int i = ctz64(U);
            U &= U - 1;
            ctx_step<PK, 0>(i, b, act);
            ctx_step<PK, 1>(i, b, act);
        }
    }

    // MRP_Encoder/Decoder :593-629
    template <int c>
    BPC_FI void mrp_step(int i, int b, bool act, uint32_t P) {
        const bool cand = act && ((s.R[c] >> i) & 1);
        if (!w.any(cand)) return;
        if (ENC) {
            ac_enc(cand, cand ? data_bit<PK_MRP>(i, c, b) : 0u, P);
        } else {
            ring_ensure();
            const uint32_t sym = ac_dec(cand, P);
            if (cand && sym && b <= 27) B[c] |= 1ull << i;
        }
    }

    BPC_FI void mrp_pass(int b, bool act) {
        const uint32_t P = act ? tab[g + b] : 0u;
        uint64_t U = warp_or64(w, act ? ((s.R[0] | s.R[1]) & G::ROWS) : 0ull);
        while (U) {
            const int i = ctz64(U);
            U &= U - 1;
            mrp_step<0>(i, b, act, P);
            mrp_step<1>(i, b, act, P);
        }
        if (act) {
            s.R[0] = s.S[0];
            s.R[1] = s.S[1];
        }
    }

    // ------------------------------------------------------ codeblock driver
    BPC_FI void run(int cb_first) {
        const int grp = lane / G::NL;
        const int cb = cb_first + grp;
        const bool ok = cb < p.ncb;
        const int cbx = ok ? cb % p.ncbx : 0, cby = ok ? cb / p.ncbx : 0;
        const int x = cbx * CBS + 2 * gl, y0 = cby * CBS;
        // Find_Subband :84-111, per lane (x of the lane, y of the block top)
        int lvl = p.levels, sb = 0;
        for (int a = 1; a <= p.levels; a++) {
            const bool hx = x >= (p.X >> a), hy = y0 >= (p.Y >> a);
            if (hx || hy) {
                lvl = a - 1;
                sb = hx ? (hy ? 2 : 0) : 1;
                break;
            }
        }
        g = lvl * 45 + sb * 15;
        for (int k = 0; k < 2; k++) s.S[k] = s.R[k] = s.N[k] = 0ull;
        s.C[0] = s.C[1] = PASSES == 3 ? G::ROWS : 0ull;  // CP flag at start (:34-39, :73-78)
        s.XL = s.XR = s.XNL = s.XNR = 0ull;
        s.lower = s.size = s.resv = s.cw = 0u;
        s.cnt = 0u;
        s.has_resv = 0;
        s.status = 0;
        const size_t cap = (size_t)G::CAP;
        const int32_t *src = p.in + (size_t)y0 * (size_t)p.X + (size_t)x;
        msb = -1;
        top = -1;
        if (ENC) {
            slot_out = p.out + (ok ? (size_t)cb * cap : 0);
            // Read_Coefficients :14-44 + Find_MSB :114-161: signs and OR
            uint32_t mx = 0;
            if (ok) {
                for (int i = 0; i < CBS; i++) {
                    int32_t v0, v1;
                    w.load2(src + (size_t)i * (size_t)p.X, v0, v1);
                    const uint32_t m0 = v0 < 0 ? 0u - (uint32_t)v0 : (uint32_t)v0;
                    const uint32_t m1 = v1 < 0 ? 0u - (uint32_t)v1 : (uint32_t)v1;
                    s.N[0] |= (uint64_t)(v0 < 0) << i;
                    s.N[1] |= (uint64_t)(v1 < 0) << i;
                    mx |= m0 | m1;
                }
            }
            if (mx >= (1u << 28)) s.status |= ST_INPUT_RANGE;
            for (int o = G::NL / 2; o; o >>= 1) mx |= w.shfl_xor(mx, o);
            if (ok) {
                msb = mx ? 31 - clz32(mx) : 32;
                if (gl == 0) slot_out[0] = msb;  // :1155
                // bitplanes 0..min(MSB, 27): transpose 32 rows x 32 bits at a time
                top = msb <= 27 ? msb : -1;
                if (top >= 0) {
#pragma unroll 1
                    for (int q = 0; q < 2 * NH; q++) {
                        const int c = q / NH, h = q % NH;
                        uint32_t a[32];
#pragma unroll
                        for (int r = 0; r < 32; r++) {
                            const int32_t v = w.load1(src + (size_t)(h * 32 + r) * (size_t)p.X + c);
                            a[r] = v < 0 ? 0u - (uint32_t)v : (uint32_t)v;
                        }
                        transpose32(a);
#pragma unroll
                        for (int k = 0; k < 28; k++)
                            if (k <= top) planes[k][c * 2 + h] = a[k];
                    }
                }
            }
            // neighbour sign columns are data: lane-1's right, lane+1's left
            const uint64_t up = shfl_up64(w, s.N[1]), dn = shfl_down64(w, s.N[0]);
            s.XNL = gl > 0 ? up : 0ull;
            s.XNR = gl < G::NL - 1 ? dn : 0ull;
        } else {
            slot_in = p.in + (ok ? (size_t)cb * cap : 0);
            if (ok) {
                ring_load(0u, G::RING);
                s.ring_hi = G::RING;
            } else {
                s.ring_hi = 0x7fffffffu;
            }
            w.sync();
            if (ok) {
                const int m = (int)ring[0];  // :1216
                // an encoder writes 0..27 (|x| < 2^28) or 32 (all-zero block)
                if ((m >= 0 && m <= 27) || m == 32)
                    msb = m;
                else
                    s.status |= ST_BAD_STREAM;
            }
        }
        // planes, aligned across the codeblocks that share the warp
        int bmax = msb;
        for (int o = 16; o; o >>= 1) {
            const int other = (int)w.shfl_xor((uint32_t)bmax, o);
            bmax = other > bmax ? other : bmax;
        }
        for (int b = bmax; b >= 0; b--) {
            // 2-pass: planes MSB..0 run SPP, MRP.  3-pass: plane MSB runs CP
            // only, planes below run SPP, MRP, CP (:986-1018).
            const bool full = PASSES == 2 ? b <= msb : b < msb;
            const bool first_cp = PASSES == 3 && b == msb;
            plane_begin(b);
            if (w.any(full)) {
                ctx_pass<PK_SPP>(b, full);
                mrp_pass(b, full);
            }
            if (PASSES == 3 && w.any(full || first_cp)) ctx_pass<PK_CP>(b, full || first_cp);
            if (b <= msb) plane_end(b);
        }
        if (ENC) {
            if (ok) {
                if (s.has_resv) {  // flush :1020
                    if (s.resv < (uint32_t)G::CAP)
                        slot_out[s.resv] = (int32_t)s.lower;
                    else
                        s.status |= ST_OVERFLOW;
                }
                // the rest of the slot keeps the -1 fill of :1284
                for (uint32_t k = s.cnt + 1u + (uint32_t)gl; k < (uint32_t)G::CAP; k += G::NL) slot_out[k] = -1;
                if (s.cnt + 1u > (uint32_t)G::CAP) s.status |= ST_OVERFLOW;
            }
        } else if (ok) {
            // Write_Coefficients :46-63: planes back to magnitudes
            top = msb == 32 ? 0 : msb;
            int32_t *dst = p.out + (size_t)y0 * (size_t)p.X + (size_t)x;
#pragma unroll 1
            for (int q = 0; q < 2 * NH; q++) {
                const int c = q / NH, h = q % NH;
                uint32_t a[32];
#pragma unroll
                for (int k = 0; k < 32; k++) a[k] = (k < 28 && k <= top) ? planes[k < 28 ? k : 0][c * 2 + h] : 0u;
                transpose32(a);
                const uint64_t neg = s.N[c] >> (32 * h);
#pragma unroll
                for (int r = 0; r < 32; r++) {
                    const int32_t m = (int32_t)a[r];
                    w.store1(dst + (size_t)(h * 32 + r) * (size_t)p.X + c, ((neg >> r) & 1) ? -m : m);
                }
            }
        }
        if (ok && p.counts && gl == 0) p.counts[cb] = (int)s.cnt;
        int st = s.status;
        for (int o = 16; o; o >>= 1) st |= (int)w.shfl_xor((uint32_t)st, o);
        if (st && lane == 0 && p.status) w.atomic_or(p.status, st);
    }
};

}  // namespace bpc
