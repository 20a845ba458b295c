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
// column).  The encoder derives whole passes from these masks bit-parallel; the
// decoder keeps the neighbour copies current with one shuffle per step in which
// some lane's coefficient became significant.  A significance context is a
// popcount of a 9-bit neighbourhood gathered from three 3-row windows, a sign
// context one read of a 256-entry table.  Magnitudes are held as bitplanes (one
// 64-bit row mask per plane and column) in a per-thread array built with an
// in-register 32x32 bit transpose; the decoder collects decoded planes the same
// way and transposes them back at the end.  Shared memory holds the LUT bytes,
// the sign-context table and, per warp, the decoder's codeword ring or the
// encoder's event-ranking words, so a decoder CTA of 4 warps fits 7 times per SM.
//
// The code is written against a small warp interface W (lane id, ballot, any,
// shuffles, syncwarp) so the same source runs as a CUDA kernel (bpc_kernels.cu)
// and, compiled for the host with one user-level context per lane, in the CPU
// tests (tests/emu/emu_warp.cpp).
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define BPC_FI __device__ __forceinline__
#define BPC_NOINLINE __device__ __noinline__
#else
#define BPC_FI inline
#define BPC_NOINLINE inline
#endif

namespace bpc {

enum : int { ST_OVERFLOW = 1, ST_BAD_STREAM = 2, ST_INPUT_RANGE = 4, ST_LUT_RANGE = 8 };
enum : int { PK_SPP = 0, PK_MRP = 1, PK_CP = 2 };

// Sign-context table of Compute_Sign_Context (:178-211), indexed by
// (class(h) * 3 + class(v)), class = 0 for 0, 1 for > 0, 2 for < 0; 3 bits each.
constexpr uint32_t kSignTab = (0u << 0) | (2u << 3) | (3u << 6) | (4u << 9) | (6u << 12) | (0u << 15) |
                              (5u << 18) | (1u << 21) | (7u << 24);

// The decoder's sign-context table: entry k for the neighbour bits
// k = sl | nl<<1 | sr<<2 | nr<<3 | su<<4 | nu<<5 | sb<<6 | nb<<7 (s = significant,
// n = negative; left, right, up, below) holds the LUT index (ctx >> 1) in bits
// 0-1 and the predicted sign (ctx & 1) in bit 2.  Threads tid, tid + n, ...
// fill it.
constexpr int kSignTableBytes = 256;
BPC_FI void build_sign_table(uint8_t *t, int tid, int n) {
    for (int k = tid; k < kSignTableBytes; k += n) {
        const int sl = k & 1, nl = (k >> 1) & 1, sr = (k >> 2) & 1, nr = (k >> 3) & 1;
        const int su = (k >> 4) & 1, nu = (k >> 5) & 1, sb = (k >> 6) & 1, nb = (k >> 7) & 1;
        const int h = sl * (1 - 2 * nl) + sr * (1 - 2 * nr), v = su * (1 - 2 * nu) + sb * (1 - 2 * nb);
        const int hc = h == 0 ? 0 : (h > 0 ? 1 : 2), vc = v == 0 ? 0 : (v > 0 ? 1 : 2);
        const uint32_t ctx = (kSignTab >> (3 * (hc * 3 + vc))) & 7u;
        t[k] = (uint8_t)((ctx >> 1) | ((ctx & 1u) << 2));
    }
}

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
    // decoder input in the compact container: codeblock k's words (MSB and
    // codewords) are in[offsets[k] .. offsets[k+1]); null = slot layout
    const long long *offsets;
    long long in_words = 0;  // compact container: its length in words (offsets outside it are damage)
    int cb_begin, cb_end;  // codeblocks [cb_begin, cb_end) of the image are coded by this launch
    // work order of a whole-image launch: warp slot k codes the codeblocks
    // starting at order[k] (null = raster order)
    const int *order = nullptr;
    // isolated decode of a work-ordered image (launch_code): heavy = 1 codes
    // the units order[0, heavy_n), one per warp slot; heavy = 2 codes the rest,
    // one unit per warp slot first and then units taken from the queue counter
    // *ctr (zeroed by the planner).  heavy = 0: the plain grid-stride walk.
    int heavy = 0, heavy_n = 0;
    int *ctr = nullptr;
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
BPC_FI int popc64(uint64_t x) {
#if defined(__CUDA_ARCH__)
    return __popcll(x);
#else
    return __builtin_popcountll(x);
#endif
}
BPC_FI void add_u64(unsigned long long *p, unsigned long long v) {
#if defined(__CUDA_ARCH__)
    atomicAdd(p, v);
#else
    *p += v;
#endif
}
BPC_FI int ctz32(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return __ffs((int)x) - 1;
#else
    return __builtin_ctz(x);
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

BPC_FI uint32_t bit64(uint64_t m, int i) { return (uint32_t)(m >> i) & 1u; }

BPC_FI uint32_t funnel_r(uint32_t lo, uint32_t hi, int n) {
#if defined(__CUDA_ARCH__)
    return __funnelshift_r(lo, hi, n);
#else
    return (uint32_t)((((uint64_t)hi << 32) | lo) >> (n & 31));
#endif
}

// Row access inside one 32-row half H of a 64-bit column mask (row i = 32H + j):
// 32-bit shifts only.  win3h gives rows i-1, i, i+1 (0 outside the block).
template <int H>
BPC_FI uint32_t win3h(uint64_t m, int j) {
    const uint32_t lo = (uint32_t)m, hi = (uint32_t)(m >> 32);
    const uint32_t t = H == 0 ? (j ? funnel_r(lo, hi, j - 1) : (lo << 1)) : (j ? (hi >> (j - 1)) : funnel_r(lo, hi, 31));
    return t & 7u;
}
template <int H>
BPC_FI uint32_t bith(uint64_t m, int j) {
    return ((H ? (uint32_t)(m >> 32) : (uint32_t)m) >> j) & 1u;
}
template <int H>
BPC_FI uint64_t maskh(uint32_t bit, int j) {
    return (uint64_t)(bit << j) << (32 * H);
}

// Interleave the low 16 bits of a (even positions) and b (odd positions):
// row j of the left column -> bit 2j, of the right column -> bit 2j+1, which
// is the scan order of one lane's two columns.
BPC_FI uint32_t spread16(uint32_t x) {
    x &= 0xFFFFu;
    x = (x | (x << 8)) & 0x00FF00FFu;
    x = (x | (x << 4)) & 0x0F0F0F0Fu;
    x = (x | (x << 2)) & 0x33333333u;
    x = (x | (x << 1)) & 0x55555555u;
    return x;
}
BPC_FI uint32_t zip16(uint64_t l, uint64_t r, int q) {
    return spread16((uint32_t)(l >> (16 * q))) | (spread16((uint32_t)(r >> (16 * q))) << 1);
}

// Per-row count (0..8) of eight 64-bit row masks, as four bit slices
// (carry-save adder tree; bit i of slice k = bit k of the count at row i).
BPC_FI void count8(const uint64_t x[8], uint64_t &c0, uint64_t &c1, uint64_t &c2, uint64_t &c3) {
    const uint64_t s1 = x[0] ^ x[1] ^ x[2], k1 = (x[0] & x[1]) | (x[2] & (x[0] ^ x[1]));
    const uint64_t s2 = x[3] ^ x[4] ^ x[5], k2 = (x[3] & x[4]) | (x[5] & (x[3] ^ x[4]));
    const uint64_t s3 = x[6] ^ x[7], k3 = x[6] & x[7];
    c0 = s1 ^ s2 ^ s3;
    const uint64_t k4 = (s1 & s2) | (s3 & (s1 ^ s2));  // weight 2
    const uint64_t t = k1 ^ k2 ^ k3, k5 = (k1 & k2) | (k3 & (k1 ^ k2));  // weight 2 / 4
    c1 = t ^ k4;
    const uint64_t k6 = t & k4;  // weight 4
    c2 = k5 ^ k6;
    c3 = k5 & k6;
}

struct Lane {
    uint64_t S[2], R[2], C[2], N[2];
    uint64_t XL, XR, XNL, XNR;
    uint32_t lower, size, resv, cw;
    uint32_t cnt;      // codewords reserved in this codeblock (group-uniform)
    uint32_t ring_hi;  // decoder: slot words [ring_hi - RING, ring_hi) are in the ring
    int status;
    // encoder: slot of the codeword left open by an earlier pass (-1: none),
    // the ev_val index the open codeword finishes into (its event in this
    // pass, or kEvOpen) and the pass's event count
    int open_slot;
    int cur_ev;
    int nev;
};

// Sizes of the encoder's per-lane event arrays.  ev_key holds one pass's
// reservations: at most one per symbol call, and a lane makes at most two
// calls per coefficient of its stripe (256 for 64x64, 128 for 32x32).  ev_val
// has one more word, the value of a codeword reserved in an earlier pass
// (kEvOpen).
constexpr int kEvKeys = 256, kEvOpen = 256, kEvVals = 257;

// Decoder codeword ring refill: lane gl of a codeblock's lane group copies
// its share of slot words [first, first + nwords) into the ring with 16-byte
// loads; words past in_cap read as -1.  Kept out of line: it runs once per 256
// codewords, and inlined into every decoder step body it would crowd the
// instruction cache.
template <int CBS>
BPC_NOINLINE void ring_fill(uint32_t *ring, const int32_t *slot_in, uint32_t in_cap, bool compact, uint32_t first,
                            int gl, int nwords) {
    constexpr int NL = CBS / 2, RING = CBS == 64 ? 512 : 256;
    const int per = nwords / NL;  // 8 or 16, multiple of 4
    for (int q = 0; q < per; q += 4) {
        const uint32_t k = first + (uint32_t)(gl * per + q);
        uint32_t v0, v1, v2, v3;
        if (k + 3 < in_cap && !compact) {
#if defined(__CUDA_ARCH__)
            const int4 v = *reinterpret_cast<const int4 *>(slot_in + k);
            v0 = (uint32_t)v.x;
            v1 = (uint32_t)v.y;
            v2 = (uint32_t)v.z;
            v3 = (uint32_t)v.w;
#else
            v0 = (uint32_t)slot_in[k];
            v1 = (uint32_t)slot_in[k + 1];
            v2 = (uint32_t)slot_in[k + 2];
            v3 = (uint32_t)slot_in[k + 3];
#endif
        } else {  // slot end, or the compact container (no 16-byte alignment)
            v0 = k + 0 < in_cap ? (uint32_t)slot_in[k + 0] : 0xFFFFFFFFu;
            v1 = k + 1 < in_cap ? (uint32_t)slot_in[k + 1] : 0xFFFFFFFFu;
            v2 = k + 2 < in_cap ? (uint32_t)slot_in[k + 2] : 0xFFFFFFFFu;
            v3 = k + 3 < in_cap ? (uint32_t)slot_in[k + 3] : 0xFFFFFFFFu;
        }
        const uint32_t r = k & (RING - 1);
        ring[r] = v0;
        ring[r + 1] = v1;
        ring[r + 2] = v2;
        ring[r + 3] = v3;
    }
}

template <class W>
BPC_FI uint64_t warp_or64(W &w, uint64_t v) {
    return ((uint64_t)w.reduce_or((uint32_t)(v >> 32)) << 32) | w.reduce_or((uint32_t)v);
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

// LAT selects the latency form of the per-lane loops, for launches whose time is
// the serial chain of their heaviest codeblocks rather than the SMs' issue rate:
// the encoder codes LAT + 1 positions per loop iteration (independent
// extractions and table reads ahead of the sequential coder updates), the
// decoder (any LAT > 0) reads a step's sign context before its significance
// decision.  They execute more instructions per symbol; the bitstream is the
// same.  LAT = 0 is the base form.
template <int PASSES, int CBS, bool ENC, class W, int LAT = 0>
struct Coder {
    using G = Geo<CBS>;
    static constexpr int NH = CBS / 32;  // 32-row halves per column
    W &w;
    const Params &p;
    Lane s;
    uint32_t *ring;        // per codeblock (decoder)
    const uint8_t *tab;    // LUT bytes
    const uint8_t *sgtab;  // decoder: sign-context table (build_sign_table)
    const int32_t *slot_in;
    int32_t *slot_out;
    uint32_t in_cap;  // decoder: words readable at slot_in (slot size, or the compact length)
    int lane, gl, g, msb;
    int top;        // highest bitplane coded from the stored planes (-1: none)
    uint32_t qtop;  // encoder: per quarter q, byte q = 1 + the highest plane stored for it (0: none)
    uint32_t gmask, ltmask;
    uint64_t B[2];  // encoder: magnitude bits of the current plane; decoder: decoded 1-bits
    int sig_base, sign_base;  // LUT byte indices of the current plane and pass
    // encoder, per pass: coded (K), symbol-1 (Y) and newly significant (NS)
    // masks, neighbour columns' significance at pass start and new in pass
    uint64_t K[2], Y[2], NS[2], XLS, XRS, XLN, XRN;
    uint64_t cs[2][4];  // context bit slices per column
    uint64_t si[2][2];  // sign-context LUT index bit slices per column
    uint64_t sg[2];     // sign symbol per column (own sign ^ predicted sign)
    uint32_t *evmask;   // per warp, 256 keys: lanes with a reservation event
    uint32_t *pfx;      // per warp, 256 keys: events before the key (ranking)
    uint8_t *ev_key;    // this lane's events of the pass: key, finished codeword
    uint32_t *ev_val;
    // bitplanes, [plane][col0 rows 0-31, col0 rows 32-63, col1 rows 0-31, col1 rows 32-63]
    // (per-thread arrays owned by the caller: an array indexed at run time
    // inside this struct would keep the whole struct out of registers)
    uint32_t (*planes)[4];

    BPC_FI Coder(W &w_, const Params &p_, uint32_t *ring_all, const uint8_t *tab_, const uint8_t *sgtab_,
                 uint32_t (*planes_)[4], uint8_t *ev_key_, uint32_t *ev_val_)
        : w(w_), p(p_), tab(tab_), sgtab(sgtab_), planes(planes_), ev_key(ev_key_), ev_val(ev_val_) {
        evmask = ring_all;
        pfx = ring_all + 256;
        lane = w.lane();
        gl = lane % G::NL;
        const int grp = lane / G::NL;
        gmask = G::NL == 32 ? 0xffffffffu : (0xffffu << (grp * 16));
        ltmask = (1u << lane) - 1u;
        ring = ring_all + grp * G::RING;
    }

    // ---------------------------------------------------------------- AC
    // Arithmetic_decoder :297-339; the codeword is read when it is reserved
    BPC_FI uint32_t ac_dec(bool act, uint32_t P) {
        const bool need = act && s.size == 0;
        const uint32_t ball = w.ballot(need);
        if (ball) {  // warp-uniform
            const uint32_t bal = ball & gmask;
            if (need) {
                // past the slot the ring holds the -1 fill; the overflow itself
                // is reported once, from the final count, at the codeblock's end
                const uint32_t idx = 1u + s.cnt + (uint32_t)popc32(bal & ltmask);
                s.cw = ring[idx & (G::RING - 1)];
                s.lower = 0;
                s.size = 0xFFFFu;
            }
            s.cnt += (uint32_t)popc32(bal);
        }
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
        ring_fill<CBS>(ring, slot_in, in_cap, p.offsets != nullptr, first, gl, nwords);
    }
    // CALLS = AC calls before the next check (each reserves at most NL
    // codewords); a refill of CHUNK words keeps [cnt+1, cnt+1+CALLS*NL) in the
    // ring for CALLS <= 4
    template <int CALLS>
    BPC_FI void ring_ensure() {
        if (s.cnt + 1u + (uint32_t)(CALLS * G::NL) > s.ring_hi) {  // group-uniform
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

    // plane registers: encoder loads the magnitude bits, decoder clears
    BPC_FI void plane_begin(int b) {
        if (ENC) {
            if (b <= top) {
                // a quarter's planes above its own highest set bit were never
                // stored: they read as zero
                const uint32_t *q = planes[b];
                const uint32_t u = (uint32_t)b;
                const uint32_t q0 = u < (qtop & 0xFFu) ? q[0] : 0u, q1 = u < ((qtop >> 8) & 0xFFu) ? q[1] : 0u;
                const uint32_t q2 = u < ((qtop >> 16) & 0xFFu) ? q[2] : 0u, q3 = u < (qtop >> 24) ? q[3] : 0u;
                B[0] = (uint64_t)q0 | ((uint64_t)q1 << 32);
                B[1] = (uint64_t)q2 | ((uint64_t)q3 << 32);
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

    // ------------------------------------------ decoder: lockstep over steps
    // The decoder cannot run ahead per lane: a context depends on what the
    // neighbour lanes decoded one step earlier, and a reservation needs the
    // number of reservations before it.  So the warp walks the steps that
    // have a candidate in some lane, all lanes together, and the rows are
    // visited per 32-row half so that every row access is a 32-bit shift.
    // One step (row 32H + j, column c), with c a constant: no selects between
    // the columns.  The step bodies (pass kind x half x column) fit the
    // instruction cache because the rare codeword-ring refill is out of line.
    template <int PK, int H, int CC>
    BPC_FI void dec_ctx_step(int j, int c_rt, int b, bool act) {
        const int c = CC >= 0 ? CC : c_rt;
        const uint64_t S0 = s.S[0], S1 = s.S[1], Sc = c ? S1 : S0;
        // the caller runs the step only if some lane has a candidate here
        const bool cand = act && (PK == PK_SPP ? !bith<H>(Sc, j) : bith<H>(c ? s.C[1] : s.C[0], j));
        const uint64_t Lm = c ? S0 : s.XL, Rm = c ? s.XR : S1;
        const uint32_t wl = win3h<H>(Lm, j), wm = win3h<H>(Sc, j), wr = win3h<H>(Rm, j);
        const uint32_t nbh = wl | ((wm & 5u) << 3) | (wr << 6);
        const uint64_t bit = maskh<H>(1u, j), bit0 = c ? 0ull : bit, bit1 = c ? bit : 0ull;
        // sign context of this coefficient (Compute_Sign_Context :178-226 over
        // l, r, u, b): one lookup in the sign-context table indexed by the
        // neighbours' bits, all decided before this step.  The latency form
        // reads it (and its probability) now, off the decision's chain.
        const uint64_t LN = c ? s.N[0] : s.XNL, MN = c ? s.N[1] : s.N[0], RN = c ? s.XNR : s.N[1];
        uint32_t se = 0, P2e = 0;
        auto sign_ctx = [&]() {
            const uint32_t nl = bith<H>(LN, j), nr = bith<H>(RN, j), wmn = win3h<H>(MN, j);
            const uint32_t sk = ((wl >> 1) & 1u) | (nl << 1) | ((wr & 2u) << 1) | (nr << 3) | ((wm & 1u) << 4) |
                                ((wmn & 1u) << 5) | ((wm & 4u) << 4) | ((wmn & 4u) << 5);
            se = sgtab[sk];
            P2e = tab[sign_base + (int)(se & 3u)];
        };
        if (LAT > 0) sign_ctx();
        bool coded = cand;
        if (PK == PK_SPP && PASSES == 3) {
            if (cand && nbh == 0) {  // SPP defers to CP (:450-452)
                s.C[0] |= bit0;
                s.C[1] |= bit1;
                coded = false;
            }
            if (!w.any(coded)) return;  // every candidate deferred
        }
        const uint32_t P = coded ? tab[sig_base + popc32(nbh)] : 0u;
        const uint32_t sym = ac_dec(coded, P);
        if (PK == PK_CP && coded) {
            s.C[0] &= ~bit0;
            s.C[1] &= ~bit1;
        }
        const bool ns = coded && sym && b <= 27;
        if (ns) {
            s.S[0] |= bit0;
            s.S[1] |= bit1;
            if (PK == PK_CP) {
                s.R[0] |= bit0;
                s.R[1] |= bit1;
            }
            B[0] |= bit0;
            B[1] |= bit1;
        }
        if (!w.any(ns)) return;
        // sign call
        if (LAT == 0) sign_ctx();
        const uint32_t pred = se >> 2;
        const uint32_t P2 = ns ? P2e : 0u;
        const uint32_t neg = (ac_dec(ns, P2) ^ pred) & 1u;
        if (ns && neg) {
            s.N[0] |= bit0;
            s.N[1] |= bit1;
        }
        // neighbour columns: lane l's column c at row i changed; lane l-1
        // (column 0) or lane l+1 (column 1) takes it over with one shuffle
        const uint32_t mine = ns ? (1u | (neg << 1)) : 0u;
        const uint32_t got = c ? w.shfl_up(mine, 1) : w.shfl_down(mine, 1);
        if (c == 0) {
            if (gl < G::NL - 1) {
                s.XR |= maskh<H>(got & 1u, j);
                s.XNR |= maskh<H>((got >> 1) & 1u, j);
            }
        } else {
            if (gl > 0) {
                s.XL |= maskh<H>(got & 1u, j);
                s.XNL |= maskh<H>((got >> 1) & 1u, j);
            }
        }
    }

    // u0 / u1: the rows of this half where some lane has a candidate in column
    // 0 / 1.  A step's candidates change only at the step itself (a coefficient
    // becomes significant, or leaves CP, when it is coded), so the pass's masks
    // taken at its start pick the steps to run, with no vote per step.
    template <int PK, int H>
    BPC_FI void dec_ctx_half(uint32_t u0, uint32_t u1, int b, bool act) {
        uint32_t u = u0 | u1;
        while (u) {
            const int j = ctz32(u);
            u &= u - 1;
            ring_ensure<4>();  // one row: two steps of up to two AC calls
            if ((u0 >> j) & 1u) dec_ctx_step<PK, H, 0>(j, 0, b, act);
            if ((u1 >> j) & 1u) dec_ctx_step<PK, H, 1>(j, 1, b, act);
        }
    }

    template <int PK>
    BPC_FI void dec_ctx_pass(int b, bool act) {
        const int off = PK == PK_CP ? p.cp_off : 0;
        sig_base = off + p.a_sig + (g + b) * 9;
        sign_base = off + p.a_sign + (g + b) * 4;
        const uint64_t c0 = act ? (PK == PK_SPP ? ~s.S[0] : s.C[0]) : 0ull;
        const uint64_t c1 = act ? (PK == PK_SPP ? ~s.S[1] : s.C[1]) : 0ull;
        const uint64_t U0 = warp_or64(w, c0 & G::ROWS), U1 = warp_or64(w, c1 & G::ROWS);
        dec_ctx_half<PK, 0>((uint32_t)U0, (uint32_t)U1, b, act);
        if (CBS == 64) dec_ctx_half<PK, 1>((uint32_t)(U0 >> 32), (uint32_t)(U1 >> 32), b, act);
    }

    // MRP_Decoder :608-629
    template <int H>
    BPC_FI void dec_mrp_step(int j, int c, int b, bool act, uint32_t P) {
        const bool cand = act && bith<H>(c ? s.R[1] : s.R[0], j);
        const uint32_t sym = ac_dec(cand, P);
        if (cand && sym && b <= 27) {
            const uint64_t bit = maskh<H>(1u, j);
            B[0] |= c ? 0ull : bit;
            B[1] |= c ? bit : 0ull;
        }
    }
    // u0 / u1 as in dec_ctx_half (the refinement set is fixed during the pass)
    template <int H>
    BPC_FI void dec_mrp_half(uint32_t u0, uint32_t u1, int b, bool act, uint32_t P) {
        uint32_t u = u0 | u1;
        while (u) {
            const int j = ctz32(u);
            u &= u - 1;
            ring_ensure<2>();  // one row: two steps of one AC call
            if ((u0 >> j) & 1u) dec_mrp_step<H>(j, 0, b, act, P);
            if ((u1 >> j) & 1u) dec_mrp_step<H>(j, 1, b, act, P);
        }
    }

    BPC_FI void dec_mrp_pass(int b, bool act) {
        const uint32_t P = act ? tab[g + b] : 0u;
        const uint64_t U0 = warp_or64(w, act ? (s.R[0] & G::ROWS) : 0ull);
        const uint64_t U1 = warp_or64(w, act ? (s.R[1] & G::ROWS) : 0ull);
        dec_mrp_half<0>((uint32_t)U0, (uint32_t)U1, b, act, P);
        if (CBS == 64) dec_mrp_half<1>((uint32_t)(U0 >> 32), (uint32_t)(U1 >> 32), b, act, P);
        if (act) {
            s.R[0] = s.S[0];
            s.R[1] = s.S[1];
        }
    }

    // ---------------------------------------------------- encoder, decoupled
    // The encoder knows every data bit up front, so per pass it computes, for
    // all rows at once, which coefficients are coded (K), which code a 1 (Y),
    // which become significant (NS) and their contexts from time-accurate
    // neighbour significance (earlier in scan order: start of pass | NS; later:
    // start of pass).  Each lane then runs its arithmetic coder over its own
    // coded symbols only.  A reservation (:268-279) is recorded as an event
    // keyed by (row, column, phase) inside a 16-row chunk; after the chunk the
    // warp ranks all events by (key, lane) -- the reference's lockstep order --
    // and the codewords go to their slots.

    // Arithmetic_encoder :261-295 for this lane, with predicated stores
    // instead of branches (lanes reserve and finish codewords at different
    // symbols, and a branch per case would serialise the warp).  A reservation
    // (:268-279) appends an event (its key; the slot is ranked at the end of
    // the pass); a finished codeword (Size == 0) stores its value with its
    // event, or in ev_val[kEvOpen] if it was reserved in an earlier pass.
    // `on` predicates the call (the optional sign call).
    BPC_FI void enc_symbol_if(bool on, uint32_t sym, uint32_t P, int key) {
        const bool rs = on && s.size == 0;
        if (rs) ev_key[s.nev] = (uint8_t)key;
        s.cur_ev = rs ? s.nev : s.cur_ev;
        s.nev += rs ? 1 : 0;
        const uint32_t size0 = rs ? 0xFFFFu : s.size, low0 = rs ? 0u : s.lower;
        const uint32_t t = ((size0 * P) >> 7) + sym;
        const uint32_t nsize = sym ? size0 - t : t;
        const uint32_t nlow = sym ? low0 + t : low0;
        const bool fin = on && nsize == 0;
        if (fin) ev_val[s.cur_ev] = nlow;
        s.size = on ? nsize : s.size;
        s.lower = on ? nlow : s.lower;
    }

    // Rank the pass's events by (key, lane) and store completed codewords.
    BPC_FI void enc_rank() {
        // The codeword left open by an earlier pass finished in this one if the
        // lane reserved again (a reservation needs Size == 0) or ends at Size 0.
        if (s.open_slot >= 0 && (s.nev > 0 || s.size == 0)) {
            if ((uint32_t)s.open_slot < (uint32_t)G::CAP)
                slot_out[s.open_slot] = (int32_t)ev_val[kEvOpen];
            else
                s.status |= ST_OVERFLOW;
            s.open_slot = -1;
        }
        if (!w.any(s.nev > 0)) return;
        for (int e = 0; e < s.nev; e++) w.smem_or(&evmask[ev_key[e]], 1u << lane);
        w.sync();
        uint32_t c[8], v = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const uint32_t m = evmask[8 * lane + k];
            c[k] = G::NL == 32 ? (uint32_t)popc32(m)
                               : ((uint32_t)popc32(m & 0xFFFFu) | ((uint32_t)popc32(m >> 16) << 16));
            v += c[k];
        }
        const uint32_t own = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = w.shfl_up(v, o);
            if (lane >= o) v += t;
        }
        uint32_t run = v - own;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            pfx[8 * lane + k] = run;
            run += c[k];
        }
        const uint32_t tot = w.shfl_idx(v, 31);
        w.sync();
        const int sh = G::NL == 32 ? 0 : 16 * (lane / G::NL);
        const uint32_t hm = G::NL == 32 ? 0xFFFFFFFFu : 0xFFFFu;
        for (int e = 0; e < s.nev; e++) {
            const int key = ev_key[e];
            const uint32_t slot = 1u + s.cnt + ((pfx[key] >> sh) & hm) + (uint32_t)popc32(evmask[key] & ltmask & gmask);
            if (e < s.nev - 1 || s.size == 0) {
                if (slot < (uint32_t)G::CAP)
                    slot_out[slot] = (int32_t)ev_val[e];
                else
                    s.status |= ST_OVERFLOW;
            } else {
                s.open_slot = (int)slot;
            }
        }
        s.cnt += (tot >> sh) & hm;
        s.cur_ev = kEvOpen;  // a codeword still open finishes into ev_val[kEvOpen]
        s.nev = 0;
        w.sync();
#pragma unroll
        for (int k = 0; k < 8; k++) evmask[8 * lane + k] = 0u;
        w.sync();
    }

    // lane-1's new right column and lane+1's new left column
    BPC_FI void enc_neighbour_ns() {
        const uint64_t up = shfl_up64(w, NS[1]), dn = shfl_down64(w, NS[0]);
        XLN = gl > 0 ? up : 0ull;
        XRN = gl < G::NL - 1 ? dn : 0ull;
    }

    // Compute_Context :164-172 for every row, with the neighbours' significance
    // as each coefficient's step sees it (Share_*_Borders :342-388).
    BPC_FI void enc_contexts() {
        const uint64_t S0 = s.S[0], S1 = s.S[1];
        const uint64_t Le = S0 | NS[0], Re = S1 | NS[1], XLe = XLS | XLN, XRe = XRS | XRN;
        uint64_t x[8];
        x[0] = XLe << 1;  // (i-1, lane-1 right)
        x[1] = Le << 1;   // (i-1, left)
        x[2] = Re << 1;   // (i-1, right)
        x[3] = XLS;       // (i, lane-1 right): later in scan
        x[4] = S1;        // (i, right): later
        x[5] = XLS >> 1;  // (i+1, *): later
        x[6] = S0 >> 1;
        x[7] = S1 >> 1;
        count8(x, cs[0][0], cs[0][1], cs[0][2], cs[0][3]);
        x[0] = Le << 1;
        x[1] = Re << 1;
        x[2] = XRe << 1;
        x[3] = Le;   // (i, left): earlier in scan
        x[4] = XRe;  // (i, lane+1 left): earlier
        x[5] = S0 >> 1;
        x[6] = S1 >> 1;
        x[7] = XRS >> 1;
        count8(x, cs[1][0], cs[1][1], cs[1][2], cs[1][3]);
    }

    // Compute_Sign_Context :178-226 for every row at once.  With pos/neg the
    // significant-positive / significant-negative neighbours, the sums
    // h = sgn(l) + sgn(r) and v = sgn(u) + sgn(b) reduce to the classes
    // h > 0 = (pl & ~nr) | (pr & ~nl), h < 0 = (nl & ~pr) | (nr & ~pl), and the
    // table of :184-208 to three boolean functions of the classes: the LUT
    // index (ctx >> 1) bits and the predicted-sign bit (ctx & 1).
    BPC_FI void enc_sign_slices() {
        const uint64_t Le = s.S[0] | NS[0], Re = s.S[1] | NS[1], XRe = XRS | XRN;
#pragma unroll
        for (int c = 0; c < 2; c++) {
            uint64_t sl, nl, sr, nr, su, nu, sb, nb;
            if (c == 0) {
                sl = XLS; nl = s.XNL;                   // (i, lane-1 right): later
                sr = s.S[1]; nr = s.N[1];               // (i, right): later
                su = Le << 1; nu = s.N[0] << 1;         // (i-1, left): earlier
                sb = s.S[0] >> 1; nb = s.N[0] >> 1;     // (i+1, left): later
            } else {
                sl = Le; nl = s.N[0];                   // (i, left): earlier
                sr = XRe; nr = s.XNR;                   // (i, lane+1 left): earlier
                su = Re << 1; nu = s.N[1] << 1;
                sb = s.S[1] >> 1; nb = s.N[1] >> 1;
            }
            const uint64_t pl = sl & ~nl, ml = sl & nl, pr = sr & ~nr, mr = sr & nr;
            const uint64_t pu = su & ~nu, mu = su & nu, pb = sb & ~nb, mb = sb & nb;
            const uint64_t hp = (pl & ~mr) | (pr & ~ml), hn = (ml & ~pr) | (mr & ~pl);
            const uint64_t vp = (pu & ~mb) | (pb & ~mu), vn = (mu & ~pb) | (mb & ~pu);
            const uint64_t h0 = ~(hp | hn), v0 = ~(vp | vn);
            si[c][0] = (h0 & ~v0) | (hp & vp) | (hn & vn);
            si[c][1] = (hp & ~vn) | (hn & ~vp);
            sg[c] = s.N[c] ^ ((h0 & vn) | hn);
        }
    }

    // Compute_Sign_Context :214-226 for a coefficient that became significant
    BPC_FI int enc_sign_ctx(int i, int c) {
        const uint64_t Le = s.S[0] | NS[0], Re = s.S[1] | NS[1];
        // c is a runtime value here: select, never index (keeps the state in registers)
        const uint64_t Me = c ? Re : Le, Ml = c ? s.S[1] : s.S[0], Nc = c ? s.N[1] : s.N[0];
        const int us = i ? (int)bit64(Me, i - 1) : 0, un = i ? (int)bit64(Nc, i - 1) : 0;
        const int bs = (int)bit64(Ml >> 1, i), bn = (int)bit64(Nc >> 1, i);
        int ls, ln, rs, rn;
        if (c == 0) {
            ls = (int)bit64(XLS, i);
            ln = (int)bit64(s.XNL, i);
            rs = (int)bit64(s.S[1], i);
            rn = (int)bit64(s.N[1], i);
        } else {
            ls = (int)bit64(Le, i);
            ln = (int)bit64(s.N[0], i);
            rs = (int)bit64(XRS | XRN, i);
            rn = (int)bit64(s.XNR, i);
        }
        const int h = ls * (1 - 2 * ln) + rs * (1 - 2 * rn);
        const int v = us * (1 - 2 * un) + bs * (1 - 2 * bn);
        const int hc = h == 0 ? 0 : (h > 0 ? 1 : 2), vc = v == 0 ? 0 : (v > 0 ? 1 : 2);
        return (int)((kSignTab >> (3 * (hc * 3 + vc))) & 7u);
    }

    // 3-pass SPP (:412-456): a non-significant coefficient is coded only if a
    // neighbour is significant when its step comes, and coding can make it
    // significant, so significance spreads within the pass.  A coefficient's
    // "dynamic" neighbours are the ones earlier in scan order, so the new
    // significance set is the least fixed point of
    //   new = PN & (static | dyn(new)),  PN = non-significant with data bit 1,
    // reached from new = PN & static in as many rounds as the longest chain.
    BPC_FI void enc_spp3_propagate(bool act, bool lowp) {
        const uint64_t S0 = s.S[0], S1 = s.S[1];
        const uint64_t dXL = XLS | (XLS << 1) | (XLS >> 1), dXR = XRS | (XRS << 1) | (XRS >> 1);
        const uint64_t dS0 = S0 | (S0 << 1) | (S0 >> 1), dS1 = S1 | (S1 << 1) | (S1 >> 1);
        const uint64_t statL = dXL | (S0 << 1) | (S0 >> 1) | dS1;
        const uint64_t statR = dS0 | (S1 << 1) | (S1 >> 1) | dXR;
        const uint64_t cand0 = act ? ~S0 & G::ROWS : 0ull, cand1 = act ? ~S1 & G::ROWS : 0ull;
        const uint64_t pn0 = lowp ? cand0 & B[0] : 0ull, pn1 = lowp ? cand1 & B[1] : 0ull;
        uint64_t ns0 = pn0 & statL, ns1 = pn1 & statR, nxl = 0, nxr = 0;
        for (;;) {
            const uint64_t up = shfl_up64(w, ns1), dn = shfl_down64(w, ns0);
            nxl = gl > 0 ? up : 0ull;
            nxr = gl < G::NL - 1 ? dn : 0ull;
            const uint64_t n0 = pn0 & (statL | ((nxl | ns0 | ns1) << 1));
            const uint64_t n1 = pn1 & (statR | ((n0 | ns1 | nxr) << 1) | n0 | nxr);
            const bool changed = (n0 != ns0) || (n1 != ns1);
            ns0 = n0;
            ns1 = n1;
            if (!w.any(changed)) break;
        }
        NS[0] = ns0;
        NS[1] = ns1;
        XLN = nxl;
        XRN = nxr;
        const uint64_t dynL = (nxl | ns0 | ns1) << 1;
        const uint64_t dynR = ((ns0 | ns1 | nxr) << 1) | ns0 | nxr;
        K[0] = cand0 & (statL | dynL);
        K[1] = cand1 & (statR | dynR);
        s.C[0] |= cand0 & ~K[0];  // deferred to CP (:450-452)
        s.C[1] |= cand1 & ~K[1];
    }

    // One pass = masks (what is coded, with which context and symbol), code
    // (the lane's arithmetic coder over those symbols, events ranked) and
    // commit (the state the next pass sees).  LUT training replaces the code
    // step with stats_pass.
    template <int PK>
    BPC_FI void enc_pass(int b, bool act) {
        enc_pass_masks<PK>(b, act);
        enc_pass_code<PK>(b, act);
        enc_pass_commit<PK>(act);
    }

    template <int PK>
    BPC_FI void enc_pass_masks(int b, bool act) {
        // The data bit coded at plane b is magnitude bit b for b <= 27; above
        // that the reference reads its flag bits (b+1 = 29 refinement, 30 CP,
        // 31 significance, >= 32 nothing), which for the coefficients each pass
        // visits are constants: MRP reads 1 at b = 28 and 30, CP reads 1 at
        // b = 29 (the CP flag itself) without the coefficient becoming
        // significant (:523-530).  Planes >= 28 only occur for MSB 32.
        const bool lowp = b <= 27;
#pragma unroll
        for (int c = 0; c < 2; c++) {
            if (PK == PK_MRP) {
                K[c] = act ? s.R[c] : 0ull;
                Y[c] = lowp ? (K[c] & B[c]) : ((b == 28 || b == 30) ? K[c] : 0ull);
                NS[c] = 0ull;
            } else if (PK == PK_CP) {
                K[c] = act ? s.C[c] : 0ull;
                NS[c] = lowp ? (K[c] & B[c]) : 0ull;
                Y[c] = lowp ? NS[c] : (b == 29 ? K[c] : 0ull);
            } else if (PASSES == 2) {
                K[c] = act ? (~s.S[c] & G::ROWS) : 0ull;
                NS[c] = lowp ? (K[c] & B[c]) : 0ull;
                Y[c] = NS[c];
            }
        }
        if (PK == PK_SPP && PASSES == 3) {
            enc_spp3_propagate(act, lowp);
            Y[0] = NS[0];
            Y[1] = NS[1];
        } else if (PK != PK_MRP) {
            enc_neighbour_ns();
        }
        if (PK != PK_MRP) {
            enc_contexts();
            enc_sign_slices();
        }
    }

    // significance context of position t from its four bit slices
    static BPC_FI uint32_t ctx4(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, int t) {
        return ((c0 >> t) & 1u) | (((c1 >> t) & 1u) << 1) | (((c2 >> t) & 1u) << 2) | (((c3 >> t) & 1u) << 3);
    }

    template <int PK>
    BPC_FI void enc_pass_code(int b, bool act) {
        const int off = PK == PK_CP ? p.cp_off : 0;
        const int sig_b = off + p.a_sig + (g + b) * 9, sign_b = off + p.a_sign + (g + b) * 4;
        const uint32_t Pref = PK == PK_MRP && act ? (uint32_t)tab[g + b] : 0u;
        // one lane's coded symbols in scan order: 16 rows at a time, the two
        // columns interleaved so that position t = 2*row + column
#pragma unroll 1
        for (int q = 0; q < CBS / 16; q++) {
            uint32_t kq = zip16(K[0], K[1], q);
            if (!kq) continue;
            const uint32_t yq = zip16(Y[0], Y[1], q);
            uint32_t nq = 0, c0 = 0, c1 = 0, c2 = 0, c3 = 0, s0 = 0, s1 = 0, gq = 0;
            if (PK != PK_MRP) {
                nq = zip16(NS[0], NS[1], q);
                c0 = zip16(cs[0][0], cs[1][0], q);
                c1 = zip16(cs[0][1], cs[1][1], q);
                c2 = zip16(cs[0][2], cs[1][2], q);
                c3 = zip16(cs[0][3], cs[1][3], q);
                s0 = zip16(si[0][0], si[1][0], q);
                s1 = zip16(si[0][1], si[1][1], q);
                gq = zip16(sg[0], sg[1], q);
            }
            if constexpr (LAT >= 2) {  // three positions per iteration, the later ones predicated
                do {
                    const int t = ctz32(kq);
                    kq &= kq - 1;
                    const bool two = kq != 0u;
                    const int t2 = two ? ctz32(kq) : t;
                    kq &= two ? kq - 1 : kq;
                    const bool three = kq != 0u;
                    const int t3 = three ? ctz32(kq) : t;
                    kq &= three ? kq - 1 : kq;
                    const int key = (32 * q + t) * 2, key2 = (32 * q + t2) * 2, key3 = (32 * q + t3) * 2;
                    if (PK == PK_MRP) {
                        enc_symbol_if(true, (yq >> t) & 1u, Pref, key);
                        enc_symbol_if(two, (yq >> t2) & 1u, Pref, key2);
                        enc_symbol_if(three, (yq >> t3) & 1u, Pref, key3);
                    } else {
                        const uint32_t ca = ctx4(c0, c1, c2, c3, t), cb2 = ctx4(c0, c1, c2, c3, t2);
                        const uint32_t cc3 = ctx4(c0, c1, c2, c3, t3);
                        const uint32_t sa = ((s0 >> t) & 1u) | (((s1 >> t) & 1u) << 1);
                        const uint32_t sb = ((s0 >> t2) & 1u) | (((s1 >> t2) & 1u) << 1);
                        const uint32_t sc = ((s0 >> t3) & 1u) | (((s1 >> t3) & 1u) << 1);
                        const uint32_t Pa = tab[sig_b + (int)ca], P2a = tab[sign_b + (int)sa];
                        const uint32_t Pb = tab[sig_b + (int)cb2], P2b = tab[sign_b + (int)sb];
                        const uint32_t Pc = tab[sig_b + (int)cc3], P2c = tab[sign_b + (int)sc];
                        enc_symbol_if(true, (yq >> t) & 1u, Pa, key);
                        enc_symbol_if(((nq >> t) & 1u) != 0u, (gq >> t) & 1u, P2a, key + 1);
                        enc_symbol_if(two, (yq >> t2) & 1u, Pb, key2);
                        enc_symbol_if(two && ((nq >> t2) & 1u) != 0u, (gq >> t2) & 1u, P2b, key2 + 1);
                        enc_symbol_if(three, (yq >> t3) & 1u, Pc, key3);
                        enc_symbol_if(three && ((nq >> t3) & 1u) != 0u, (gq >> t3) & 1u, P2c, key3 + 1);
                    }
                } while (kq);
            } else if constexpr (LAT == 1) {  // two positions per iteration, the second predicated
                do {
                    const int t = ctz32(kq);
                    kq &= kq - 1;
                    const bool two = kq != 0u;
                    const int t2 = two ? ctz32(kq) : t;
                    kq &= two ? kq - 1 : kq;
                    const int key = (32 * q + t) * 2, key2 = (32 * q + t2) * 2;
                    if (PK == PK_MRP) {
                        enc_symbol_if(true, (yq >> t) & 1u, Pref, key);
                        enc_symbol_if(two, (yq >> t2) & 1u, Pref, key2);
                    } else {
                        const uint32_t ca = ctx4(c0, c1, c2, c3, t), cb2 = ctx4(c0, c1, c2, c3, t2);
                        const uint32_t sa = ((s0 >> t) & 1u) | (((s1 >> t) & 1u) << 1);
                        const uint32_t sb = ((s0 >> t2) & 1u) | (((s1 >> t2) & 1u) << 1);
                        const uint32_t Pa = tab[sig_b + (int)ca], P2a = tab[sign_b + (int)sa];
                        const uint32_t Pb = tab[sig_b + (int)cb2], P2b = tab[sign_b + (int)sb];
                        enc_symbol_if(true, (yq >> t) & 1u, Pa, key);
                        enc_symbol_if(((nq >> t) & 1u) != 0u, (gq >> t) & 1u, P2a, key + 1);
                        enc_symbol_if(two, (yq >> t2) & 1u, Pb, key2);
                        enc_symbol_if(two && ((nq >> t2) & 1u) != 0u, (gq >> t2) & 1u, P2b, key2 + 1);
                    }
                } while (kq);
            } else {
                do {
                    const int t = ctz32(kq);
                    kq &= kq - 1;
                    const int key = (32 * q + t) * 2;  // (row, column, phase) in the pass
                    if (PK == PK_MRP) {
                        enc_symbol_if(true, (yq >> t) & 1u, Pref, key);
                    } else {
                        const uint32_t ctx = ctx4(c0, c1, c2, c3, t);
                        enc_symbol_if(true, (yq >> t) & 1u, tab[sig_b + (int)ctx], key);
                        // the sign call of a coefficient that became significant
                        const uint32_t sidx = ((s0 >> t) & 1u) | (((s1 >> t) & 1u) << 1);
                        enc_symbol_if(((nq >> t) & 1u) != 0u, (gq >> t) & 1u, tab[sign_b + (int)sidx], key + 1);
                    }
                } while (kq);
            }
        }
        enc_rank();
    }

    template <int PK>
    BPC_FI void enc_pass_commit(bool act) {
        if (PK == PK_MRP) {
            if (act) {
                s.R[0] = s.S[0];
                s.R[1] = s.S[1];
            }
        } else {
            s.S[0] |= NS[0];
            s.S[1] |= NS[1];
            XLS |= XLN;
            XRS |= XRN;
            if (PK == PK_CP) {
                s.R[0] |= NS[0];
                s.R[1] |= NS[1];
                s.C[0] &= ~K[0];
                s.C[1] &= ~K[1];
            }
        }
    }

    // LUT training (no counterpart in the reference, whose tables come
    // pre-trained): for every LUT entry the pass uses, the number of symbols
    // coded with it and how many of them were 1, counted bit-parallel from
    // the pass masks.  Planes 0..14 only -- the planes of the LUT files, where
    // each entry belongs to exactly one (level, subband, plane, context).
    BPC_FI void tally(unsigned long long *st, int idx, uint32_t n, uint32_t ones) {
        if (n) add_u64(st + 2 * idx, n);
        if (ones) add_u64(st + 2 * idx + 1, ones);
    }
    template <int PK>
    BPC_FI void stats_pass(int b, bool act, unsigned long long *st) {
        if (!act || b >= 15) return;
        const int off = PK == PK_CP ? p.cp_off : 0;
        if (PK == PK_MRP) {
            tally(st, g + b, (uint32_t)(popc64(K[0]) + popc64(K[1])), (uint32_t)(popc64(Y[0]) + popc64(Y[1])));
        } else {
            stats_ctx(st, off, b);
        }
    }
    BPC_FI void stats_ctx(unsigned long long *st, int off, int b) {
#pragma unroll 1
        for (int k = 0; k < 9; k++) {
            uint32_t n = 0, ones = 0;
#pragma unroll
            for (int c = 0; c < 2; c++) {
                uint64_t m = K[c];
#pragma unroll
                for (int q = 0; q < 4; q++) m &= ((k >> q) & 1) ? cs[c][q] : ~cs[c][q];
                n += (uint32_t)popc64(m);
                ones += (uint32_t)popc64(m & Y[c]);
            }
            tally(st, off + p.a_sig + (g + b) * 9 + k, n, ones);
        }
#pragma unroll 1
        for (int k = 0; k < 4; k++) {
            uint32_t n = 0, ones = 0;
#pragma unroll
            for (int c = 0; c < 2; c++) {
                const uint64_t m = NS[c] & ((k & 1) ? si[c][0] : ~si[c][0]) & ((k & 2) ? si[c][1] : ~si[c][1]);
                n += (uint32_t)popc64(m);
                ones += (uint32_t)popc64(m & sg[c]);
            }
            tally(st, off + p.a_sign + (g + b) * 4 + k, n, ones);
        }
    }
    template <int PK>
    BPC_FI void train_pass(int b, bool act, unsigned long long *st) {
        enc_pass_masks<PK>(b, act);
        stats_pass<PK>(b, act, st);
        enc_pass_commit<PK>(act);
    }

    // ------------------------------------------------------ codeblock driver
    // STATS (encoder only): gather LUT training counts into `stats` instead of
    // writing the slot stream.
    template <bool STATS = false>
    BPC_FI void run(int cb_first, unsigned long long *stats = nullptr) {
        const int grp = lane / G::NL;
        const int cb = cb_first + grp;
        const bool ok = cb < p.cb_end;
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
        s.status = 0;
        s.open_slot = -1;
        s.cur_ev = kEvOpen;
        s.nev = 0;
        XLS = XRS = XLN = XRN = 0ull;
        if (ENC) {
            for (int k = 0; k < 8; k++) evmask[8 * lane + k] = 0u;
            w.sync();
        }
        const size_t cap = (size_t)G::CAP;
        const int32_t *src = p.in + (size_t)y0 * (size_t)p.X + (size_t)x;
        msb = -1;
        top = -1;
        if (ENC) {
            slot_out = p.out + (ok ? (size_t)cb * cap : 0);
            // Read_Coefficients :14-44 + Find_MSB :114-161 in one read: per
            // 32-row half, one 8-byte load per row gives the lane's two
            // columns; signs go to N, magnitudes through a 32x32 bit
            // transpose to bitplanes 0..27 (those up to the quarter's own
            // highest set bit are stored)
            uint32_t mx = 0;
            qtop = 0u;
            if (ok) {
#pragma unroll 1
                for (int h = 0; h < NH; h++) {
                    uint32_t a0[32], a1[32], o0 = 0, o1 = 0, n0 = 0, n1 = 0;
#pragma unroll
                    for (int r = 0; r < 32; r++) {
                        int32_t v0, v1;
                        w.load2(src + (size_t)(h * 32 + r) * (size_t)p.X, v0, v1);
                        a0[r] = v0 < 0 ? 0u - (uint32_t)v0 : (uint32_t)v0;
                        a1[r] = v1 < 0 ? 0u - (uint32_t)v1 : (uint32_t)v1;
                        n0 |= (uint32_t)(v0 < 0) << r;
                        n1 |= (uint32_t)(v1 < 0) << r;
                        o0 |= a0[r];
                        o1 |= a1[r];
                    }
                    s.N[0] |= (uint64_t)n0 << (32 * h);
                    s.N[1] |= (uint64_t)n1 << (32 * h);
                    mx |= o0 | o1;
                    const int t0 = o0 ? 31 - clz32(o0) : -1, t1 = o1 ? 31 - clz32(o1) : -1;
                    qtop |= (uint32_t)(t0 + 1) << (8 * h) | (uint32_t)(t1 + 1) << (8 * (2 + h));
                    transpose32(a0);
#pragma unroll
                    for (int k = 0; k < 28; k++)
                        if (k <= t0) planes[k][h] = a0[k];
                    transpose32(a1);
#pragma unroll
                    for (int k = 0; k < 28; k++)
                        if (k <= t1) planes[k][2 + h] = a1[k];
                }
            }
            if (mx >= (1u << 28)) s.status |= ST_INPUT_RANGE;
            for (int o = G::NL / 2; o; o >>= 1) mx |= w.shfl_xor(mx, o);
            if (ok) {
                msb = mx ? 31 - clz32(mx) : 32;
                if (gl == 0 && !STATS) slot_out[0] = msb;  // :1155
                top = msb <= 27 ? msb : -1;  // planes >= 28 are flag bits, not magnitudes
            }
            // neighbour sign columns are data: lane-1's right, lane+1's left
            const uint64_t up = shfl_up64(w, s.N[1]), dn = shfl_down64(w, s.N[0]);
            s.XNL = gl > 0 ? up : 0ull;
            s.XNR = gl < G::NL - 1 ? dn : 0ull;
        } else {
            if (p.offsets) {  // compact container; words past the codeblock read as the -1 fill
                const long long o0 = ok ? p.offsets[cb] : 0, o1 = ok ? p.offsets[cb + 1] : 0;
                // damaged offsets (outside the container, or decreasing) read
                // nothing: the codeblock then decodes as a bad stream
                const bool inside = o0 >= 0 && o1 >= o0 && o1 <= p.in_words;
                slot_in = p.in + (inside ? o0 : 0);
                const long long n = inside ? o1 - o0 : 0;
                in_cap = (uint32_t)(n > (long long)cap ? (long long)cap : n);
            } else {
                slot_in = p.in + (ok ? (size_t)cb * cap : 0);
                in_cap = (uint32_t)cap;
            }
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
            if (ENC && STATS) {
                if (w.any(full)) {
                    train_pass<PK_SPP>(b, full, stats);
                    train_pass<PK_MRP>(b, full, stats);
                }
                if (PASSES == 3 && w.any(full || first_cp)) train_pass<PK_CP>(b, full || first_cp, stats);
            } else if (ENC) {
                if (w.any(full)) {
                    enc_pass<PK_SPP>(b, full);
                    enc_pass<PK_MRP>(b, full);
                }
                if (PASSES == 3 && w.any(full || first_cp)) enc_pass<PK_CP>(b, full || first_cp);
            } else {
                if (w.any(full)) {
                    dec_ctx_pass<PK_SPP>(b, full);
                    dec_mrp_pass(b, full);
                }
                if (PASSES == 3 && w.any(full || first_cp)) dec_ctx_pass<PK_CP>(b, full || first_cp);
            }
            if (b <= msb) plane_end(b);
        }
        if (ENC) {
            if (ok && !STATS) {
                if (s.size != 0) {  // flush :1020 (a finished codeword is already stored)
                    if ((uint32_t)s.open_slot < (uint32_t)G::CAP)
                        slot_out[s.open_slot] = (int32_t)s.lower;
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
                const uint64_t neg = (c ? s.N[1] : s.N[0]) >> (32 * h);
#pragma unroll
                for (int r = 0; r < 32; r++) {
                    const int32_t m = (int32_t)a[r];
                    w.store1(dst + (size_t)(h * 32 + r) * (size_t)p.X + c, ((neg >> r) & 1) ? -m : m);
                }
            }
        }
        if (!ENC && ok && s.cnt >= (uint32_t)G::CAP) s.status |= ST_OVERFLOW;  // a reservation read past the slot
        if (ok && p.counts && gl == 0) p.counts[cb] = (int)s.cnt;
        int st = s.status;
        for (int o = 16; o; o >>= 1) st |= (int)w.shfl_xor((uint32_t)st, o);
        if (st && lane == 0 && p.status) w.atomic_or(p.status, st);
    }
};

}  // namespace bpc
