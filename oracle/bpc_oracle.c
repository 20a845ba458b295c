/*
 * bpc_oracle.c -- CPU restatement of the BPC-PaCo codeblock coder.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the CUDA product path is
 * compared against (tests/, __graft_entry__.smoke(), bench.py's cpu_baseline and
 * --impl reference arm).  It is never linked into, loaded by or called from the
 * product library.
 *
 * It restates, scalar and in plain C, the algorithm of the reference
 * PabloEnfedaque/CUDA_BPC-PaCo:
 *   source/BPC_PaCo.cu:14-1224   device coder (loader, MSB, contexts, AC, passes)
 *   source/main_example.cu:219-448 load_LUTs (LUT text format)
 *
 * Warp semantics.  The reference runs one warp per codeblock and relies on
 * pre-Volta lockstep execution: inside each coefficient step every lane first
 * makes its significance/refinement arithmetic-coder call, then every lane that
 * coded a 1 makes its sign call (BPC_PaCo.cu:412-456).  A lane whose interval
 * is exhausted reserves the next codeword slot with __ballot + __popc, so slots
 * are handed out in ascending lane order within a call site
 * (BPC_PaCo.cu:268-279).  Here that is a sequential lane loop per phase with a
 * plain counter.  Lanes of one step never touch each other's neighbourhoods
 * (they are two columns apart), so sequential lanes equal the lockstep
 * snapshot.
 *
 * Defined behaviour where the reference is undefined (documented per case):
 *   - shifts by >= 32 give 0 (PTX shr/shl clamp), e.g. MSB = 32 for an
 *     all-zero codeblock (BPC_PaCo.cu:159) and the data-bit reads at b+1 >= 32;
 *   - LUT reads past the loaded array read 0 (the device LUT is the loader
 *     array zero-padded);
 *   - codewords that would land beyond the codeblock's slot are dropped and
 *     the codeblock is flagged BPCO_ST_OVERFLOW (the reference writes into the
 *     next slot, BPC_PaCo.cu:292);
 *   - decoder reads beyond the slot return 0xFFFFFFFF (the -1 fill) and flag
 *     BPCO_ST_OVERFLOW; an MSB word outside {0..27, 32} (no encoder writes
 *     28..31 for inputs |x| < 2^28) decodes to zeros and flags
 *     BPCO_ST_BAD_STREAM.
 * Codeblocks of 32x32 (not expressible in the reference, CBLOCK_WIDTH is wired
 * to 2*WARPSIZE in common.h:49-51) use 16 lanes x 2 columns x 32 rows, borders
 * at group lanes 0/15, a 1024-int slot at the codeblock's raster index.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

#define BPCO_OK 0
#define BPCO_ERR_ARG -1
#define BPCO_ERR_FILE -2
#define BPCO_ERR_PARSE -3
#define BPCO_ERR_CAP -4

#define BPCO_ST_OVERFLOW 1
#define BPCO_ST_BAD_STREAM 2
#define BPCO_ST_INPUT_RANGE 4

/* common.h:29-35 */
#define NBP 15 /* LUT_N_BITPLANES */
#define NSB 3  /* LUT_N_SUBBANDS */
#define NCTX_REF 1
#define NCTX_SIGN 4
#define NCTX_SIG 9

#define SIGMA (1u << 31)
#define CPF (1u << 30)
#define REFF (1u << 29)

static inline uint32_t shr32(uint32_t x, int n) { return (n >= 32 || n < 0) ? 0u : (x >> n); }
static inline uint32_t shl32(uint32_t x, int n) { return (n >= 32 || n < 0) ? 0u : (x << n); }

/* ------------------------------------------------------------------------- */
/* LUT loader: main_example.cu:219-448                                        */
/* ------------------------------------------------------------------------- */

typedef struct {
    char *buf;
    size_t len, pos;
} scanner;

static int read_file(const char *path, scanner *s) {
    FILE *f = fopen(path, "rb");
    if (!f) return BPCO_ERR_FILE;
    fseek(f, 0, SEEK_END);
    long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    s->buf = (char *)malloc((size_t)n + 1);
    if (!s->buf) { fclose(f); return BPCO_ERR_FILE; }
    size_t got = fread(s->buf, 1, (size_t)n, f);
    fclose(f);
    s->buf[got] = 0;
    s->len = got;
    s->pos = 0;
    return BPCO_OK;
}

static void skip_ws(scanner *s) {
    while (s->pos < s->len && (s->buf[s->pos] == ' ' || s->buf[s->pos] == '\n' || s->buf[s->pos] == '\r' ||
                               s->buf[s->pos] == '\t'))
        s->pos++;
}

/* returns 1 on a parsed int, 0 at end of input, -1 on garbage */
static int next_int(scanner *s, long *v) {
    skip_ws(s);
    if (s->pos >= s->len) return 0;
    char *end = NULL;
    long x = strtol(s->buf + s->pos, &end, 10);
    if (end == s->buf + s->pos) return -1;
    s->pos = (size_t)(end - s->buf);
    *v = x;
    return 1;
}

static int expect_colon(scanner *s) {
    skip_ws(s);
    if (s->pos < s->len && s->buf[s->pos] == ':') { s->pos++; return 1; }
    return 0;
}

/* One record "lvl sb bp : v0 .. v(n-1)".  1 = record, 0 = clean EOF, <0 error. */
static int next_record(scanner *s, int nvals, int *bp, int *vals) {
    long a, b, c, v;
    int r = next_int(s, &a);
    if (r == 0) return 0;
    if (r < 0) return BPCO_ERR_PARSE;
    if (next_int(s, &b) != 1 || next_int(s, &c) != 1 || !expect_colon(s)) return BPCO_ERR_PARSE;
    for (int k = 0; k < nvals; k++) {
        if (next_int(s, &v) != 1) return BPCO_ERR_PARSE;
        vals[k] = (int)v;
    }
    *bp = (int)c;
    return 1;
}

/* Writes past the allocation are dropped (the reference overflows its heap
 * buffer when DWT_LEVELS is smaller than the file's group count). */
static inline void lut_put(int *lut, int total, long idx, int v) {
    if (idx >= 0 && idx < total) lut[idx] = v;
}

/* Parse one section file into lut[base ..] following main_example.cu:285-300
 * (ref), :309-335 (sig), :341-364 (sign), :369-426 (cp_sig/cp_sign): a new
 * (level, subband) group starts when the bitplane column does not increase; the
 * previous group is then filled with 64 from entry prev*N+1 to the end of its
 * max_bitplane*N span (this also overwrites contexts 1..N-1 of the last listed
 * bitplane), and the write cursor advances by max_bitplane*N. */
static int load_section(const char *path, int nctx, int mb, int *lut, int total, long base) {
    scanner s;
    int rc = read_file(path, &s);
    if (rc) return rc;
    long i = base;
    int prev = -1, bp = 0, vals[NCTX_SIG];
    for (;;) {
        int r = next_record(&s, nctx, &bp, vals);
        if (r == 0) break;
        if (r < 0) { free(s.buf); return r; }
        if (bp <= prev) {
            for (long z = 0; z < (long)(mb - prev) * nctx; z++) lut_put(lut, total, i + (long)prev * nctx + z + 1, 64);
            i += (long)mb * nctx;
        }
        prev = bp;
        for (int k = 0; k < nctx; k++) lut_put(lut, total, i + (long)bp * nctx + k, vals[k]);
    }
    free(s.buf);
    return BPCO_OK;
}

static int scan_max_bitplane(const char *path, int nctx, int *maxbp) {
    scanner s;
    int rc = read_file(path, &s);
    if (rc) return rc;
    int bp, vals[NCTX_SIG];
    for (;;) {
        int r = next_record(&s, nctx, &bp, vals);
        if (r == 0) break;
        if (r < 0) { free(s.buf); return r; }
        if (bp > *maxbp) *maxbp = bp;
    }
    free(s.buf);
    return BPCO_OK;
}

/* Size in ints of the loader's array for (max_bitplane, levels, passes):
 * main_example.cu:266-278. */
static long lut_total(int mb, int levels, int passes) {
    long ref_n = (long)NSB * mb * NCTX_REF * levels + (long)mb * NCTX_REF;
    long sig_n = (long)NSB * mb * NCTX_SIG * levels + (long)mb * NCTX_SIG;
    long sign_n = (long)NSB * mb * NCTX_SIGN * levels + (long)mb * NCTX_SIGN;
    return passes == 3 ? ref_n + 2 * sig_n + 2 * sign_n : ref_n + sig_n + sign_n;
}

int bpco_load_luts(const char *folder, int passes, int levels, int *out, int cap, int *n_out) {
    if (!folder || (passes != 2 && passes != 3) || levels < 1 || levels > 12) return BPCO_ERR_ARG;
    char path[4096];
    int mb = -1, rc;
    const char *names[5] = {"ref.txt", "sig.txt", "sign.txt", "cp_sig.txt", "cp_sign.txt"};
    const int nctx[5] = {NCTX_REF, NCTX_SIG, NCTX_SIGN, NCTX_SIG, NCTX_SIGN};
    /* max bitplane over ref/sig/sign only (main_example.cu:231-264) */
    for (int f = 0; f < 3; f++) {
        snprintf(path, sizeof path, "%s%s", folder, names[f]);
        if ((rc = scan_max_bitplane(path, nctx[f], &mb))) return rc;
    }
    mb++;
    long total = lut_total(mb, levels, passes);
    if (n_out) *n_out = (int)total;
    if (!out) return BPCO_OK; /* size query */
    if (total > cap) return BPCO_ERR_CAP;
    memset(out, 0, (size_t)total * sizeof(int));
    long ref_n = (long)NSB * mb * NCTX_REF * levels + (long)mb * NCTX_REF;
    long sig_n = (long)NSB * mb * NCTX_SIG * levels + (long)mb * NCTX_SIG;
    long sign_n = (long)NSB * mb * NCTX_SIGN * levels + (long)mb * NCTX_SIGN;
    long bases[5] = {0, ref_n, ref_n + sig_n, ref_n + sig_n + sign_n, ref_n + 2 * sig_n + sign_n};
    int nfiles = passes == 3 ? 5 : 3;
    for (int f = 0; f < nfiles; f++) {
        snprintf(path, sizeof path, "%s%s", folder, names[f]);
        if ((rc = load_section(path, nctx[f], mb, out, (int)total, bases[f]))) return rc;
    }
    return BPCO_OK;
}

/* ------------------------------------------------------------------------- */
/* Codeblock geometry and LUT addressing                                       */
/* ------------------------------------------------------------------------- */

/* Find_Subband, BPC_PaCo.cu:84-111.  level 0 is the finest; LL gets (levels, 0);
 * HL = 0 (x only), LH = 1 (y only), HH = 2. */
void bpco_find_subband(int x, int y, int X, int Y, int levels, int *level, int *subband) {
    for (int aux = 1;; aux++) {
        if (aux == levels + 1) { *level = levels; *subband = 0; return; }
        int hx = x >= (X >> aux), hy = y >= (Y >> aux);
        if (hx || hy) {
            *level = aux - 1;
            *subband = hx ? (hy ? 2 : 0) : 1;
            return;
        }
    }
}

typedef struct {
    long ref, sig, sign, cp_off;
} lut_ptrs;

/* Initialize_LUT_pointers BPC_PaCo.cu:228-250 evaluated at plane b (the
 * reference decrements the pointers by N per plane, :253-258); the 3-pass CP
 * sections sit a fixed offset further (:988-989). */
static lut_ptrs lut_at_plane(int level, int sb, int b, int levels) {
    lut_ptrs p;
    long aux = (long)NSB * NBP * NCTX_REF * levels + NBP * NCTX_REF;
    p.ref = (long)level * NSB * NBP * NCTX_REF + (long)sb * NBP * NCTX_REF + (long)b * NCTX_REF;
    p.sig = (long)level * NSB * NBP * NCTX_SIG + (long)sb * NBP * NCTX_SIG + (long)b * NCTX_SIG + aux;
    aux += (long)NSB * NBP * NCTX_SIG * levels + NBP * NCTX_SIG;
    p.sign = (long)level * NSB * NBP * NCTX_SIGN + (long)sb * NBP * NCTX_SIGN + (long)b * NCTX_SIGN + aux;
    p.cp_off = (long)NSB * NBP * NCTX_SIG * levels + NBP * NCTX_SIG + (long)NSB * NBP * NCTX_SIGN * levels +
               NBP * NCTX_SIGN;
    return p;
}

/* ------------------------------------------------------------------------- */
/* Per-codeblock coder state                                                   */
/* ------------------------------------------------------------------------- */

#define MAXL 32
#define MAXR 64

typedef struct {
    int passes, levels, H, W, nl; /* rows, cols, lanes */
    const int *lut;
    long lut_n;
    int32_t *stream;      /* encoder: slot base; decoder: read-only slot base */
    const int32_t *instr; /* decoder input slot */
    long cap;             /* slot size in ints */
    uint32_t T[MAXL][2 * MAXR];
    int lvl[MAXL], sb[MAXL];
    /* arithmetic coder state per lane */
    uint32_t lower[MAXL], size[MAXL], resv[MAXL], cw[MAXL];
    int has_resv[MAXL];
    long counter;
    int status;
    int ref_quirk; /* decoder follows the reference decoder exactly */
    uint64_t *stats; /* LUT training counts, or NULL */
    long stats_n;
} cbstate;

static inline int lut_get(const cbstate *c, long idx) { return (idx >= 0 && idx < c->lut_n) ? c->lut[idx] : 0; }

/* LUT training counts (no counterpart in the reference): per LUT entry, the
 * symbols coded with it and how many were 1, for planes 0..14 (the planes of
 * the LUT files, where each entry belongs to one level/subband/plane/context). */
static inline void tally(cbstate *c, long idx, uint32_t sym, int b) {
    if (c->stats && b < NBP && idx >= 0 && idx < c->stats_n) {
        c->stats[2 * idx]++;
        c->stats[2 * idx + 1] += sym;
    }
}

/* Neighbour word at (row, global column) of the codeblock, 0 outside: the
 * shuffles of Share_{Left,Right}_Borders (:342-388) plus the zeroing of row 0 /
 * last row in the launchers (:646-704) and Correct_CB_borders at lanes 0 / last
 * (:390-410). */
static inline uint32_t nb(const cbstate *c, int r, int gc) {
    if (r < 0 || r >= c->H || gc < 0 || gc >= c->W) return 0;
    return c->T[gc >> 1][2 * r + (gc & 1)];
}

/* Compute_Context :164-172 over the 8-neighbourhood */
static inline int sig_context(const cbstate *c, int r, int gc) {
    int n = 0;
    for (int dr = -1; dr <= 1; dr++)
        for (int dc = -1; dc <= 1; dc++)
            if (dr || dc) n += (int)(nb(c, r + dr, gc + dc) >> 31);
    return n;
}

static inline int any_sig_neighbour(const cbstate *c, int r, int gc) { return sig_context(c, r, gc) != 0; }

/* Compute_Sign_Context :178-226 */
static inline int sgn_of(uint32_t w) { return (w >> 31) == 0 ? 0 : ((w & 1) ? -1 : 1); }
static int sign_context(const cbstate *c, int r, int gc) {
    int h = sgn_of(nb(c, r, gc - 1)) + sgn_of(nb(c, r, gc + 1));
    int v = sgn_of(nb(c, r - 1, gc)) + sgn_of(nb(c, r + 1, gc));
    if (h == 0) return v == 0 ? 0 : (v > 0 ? 2 : 3);
    if (h > 0) return v == 0 ? 4 : (v > 0 ? 6 : 0);
    return v == 0 ? 5 : (v > 0 ? 1 : 7);
}

/* Arithmetic_encoder :261-295.  The reservation happens when the interval is
 * exhausted at the start of a call; callers visit lanes in ascending order. */
static void ac_encode(cbstate *c, int l, uint32_t sym, int P) {
    if (c->size[l] == 0) {
        c->lower[l] = 0;
        c->size[l] = (1u << 16) - 1;
        c->resv[l] = (uint32_t)(1 + c->counter);
        c->has_resv[l] = 1;
        c->counter++;
    }
    uint32_t t = ((c->size[l] * (uint32_t)P) >> 7) + sym;
    if (sym == 0)
        c->size[l] = t;
    else {
        c->size[l] -= t;
        c->lower[l] += t;
    }
    if (c->size[l] == 0) {
        if ((long)c->resv[l] < c->cap)
            c->stream[c->resv[l]] = (int32_t)c->lower[l];
        else
            c->status |= BPCO_ST_OVERFLOW;
    }
}

/* Arithmetic_decoder :297-339 */
static uint32_t ac_decode(cbstate *c, int l, int P) {
    if (c->size[l] == 0) {
        c->lower[l] = 0;
        c->size[l] = (1u << 16) - 1;
        long idx = 1 + c->counter;
        c->counter++;
        if (idx < c->cap)
            c->cw[l] = (uint32_t)c->instr[idx];
        else {
            c->cw[l] = 0xFFFFFFFFu;
            c->status |= BPCO_ST_OVERFLOW;
        }
    }
    uint32_t t = ((c->size[l] * (uint32_t)P) >> 7) + 1;
    uint32_t thr = c->lower[l] + t;
    if (c->cw[l] >= thr) {
        c->size[l] -= t;
        c->lower[l] = thr;
        return 1;
    }
    c->size[l] = t - 1;
    return 0;
}

/* ---------------------------- encoder passes ----------------------------- */

/* SPP_Encoder :412-456; returns 1 when a sign call follows in this step */
static int spp_enc_sig(cbstate *c, int l, int r, int col, int b, int *sctx) {
    uint32_t *w = &c->T[l][2 * r + col];
    int gc = 2 * l + col;
    if (*w >> 31) return 0;
    if (c->passes == 3 && !any_sig_neighbour(c, r, gc)) {
        *w |= CPF;
        return 0;
    }
    lut_ptrs p = lut_at_plane(c->lvl[l], c->sb[l], b, c->levels);
    int ctx = sig_context(c, r, gc);
    tally(c, p.sig + ctx, shr32(*w, b + 1) & 1, b);
    ac_encode(c, l, shr32(*w, b + 1) & 1, lut_get(c, p.sig + ctx));
    if ((shr32(*w, b + 1) & 1) == 1) {
        *w |= SIGMA;
        *sctx = sign_context(c, r, gc);
        return 1;
    }
    return 0;
}

/* CP_Encoder :510-544.  The data bit is re-read after the CP flag is cleared
 * (:528-530), which only differs from the coded symbol when b + 1 == 30. */
static int cp_enc_sig(cbstate *c, int l, int r, int col, int b, int *sctx) {
    uint32_t *w = &c->T[l][2 * r + col];
    int gc = 2 * l + col;
    if (!((*w >> 30) & 1)) return 0;
    lut_ptrs p = lut_at_plane(c->lvl[l], c->sb[l], b, c->levels);
    int ctx = sig_context(c, r, gc);
    tally(c, p.sig + p.cp_off + ctx, shr32(*w, b + 1) & 1, b);
    ac_encode(c, l, shr32(*w, b + 1) & 1, lut_get(c, p.sig + p.cp_off + ctx));
    *w &= ~CPF;
    if ((shr32(*w, b + 1) & 1) == 1) {
        *w |= SIGMA | REFF;
        *sctx = sign_context(c, r, gc);
        return 1;
    }
    return 0;
}

static void enc_sign(cbstate *c, int l, int r, int col, int b, int sctx, int cp) {
    uint32_t w = c->T[l][2 * r + col];
    lut_ptrs p = lut_at_plane(c->lvl[l], c->sb[l], b, c->levels);
    long base = p.sign + (cp ? p.cp_off : 0);
    tally(c, base + (sctx >> 1), ((w & 1) == (uint32_t)(sctx & 1)) ? 0u : 1u, b);
    ac_encode(c, l, ((w & 1) == (uint32_t)(sctx & 1)) ? 0u : 1u, lut_get(c, base + (sctx >> 1)));
}

/* MRP_Encoder :593-605 */
static void mrp_enc(cbstate *c, int l, int r, int col, int b, long idx) {
    uint32_t *w = &c->T[l][2 * r + col];
    if ((*w >> 29) & 1) {
        tally(c, idx, shr32(*w, b + 1) & 1, b);
        ac_encode(c, l, shr32(*w, b + 1) & 1, lut_get(c, idx));
    }
    else if (*w >> 31)
        *w |= REFF;
}

/* The launchers :633-962 visit row 0..H-1, left column then right column; in
 * each step all lanes make their first call, then the sign calls follow. */
static void enc_ctx_pass(cbstate *c, int b, int cp) {
    int pend[MAXL], sctx[MAXL];
    for (int r = 0; r < c->H; r++)
        for (int col = 0; col < 2; col++) {
            for (int l = 0; l < c->nl; l++)
                pend[l] = cp ? cp_enc_sig(c, l, r, col, b, &sctx[l]) : spp_enc_sig(c, l, r, col, b, &sctx[l]);
            for (int l = 0; l < c->nl; l++)
                if (pend[l]) enc_sign(c, l, r, col, b, sctx[l], cp);
        }
}

static void enc_mrp_pass(cbstate *c, int b) {
    for (int r = 0; r < c->H; r++)
        for (int col = 0; col < 2; col++)
            for (int l = 0; l < c->nl; l++) {
                lut_ptrs p = lut_at_plane(c->lvl[l], c->sb[l], b, c->levels);
                mrp_enc(c, l, r, col, b, p.ref);
            }
}

/* ---------------------------- decoder passes ----------------------------- */

/* SPP_Decoder :458-507 */
static int spp_dec_sig(cbstate *c, int l, int r, int col, int b, uint32_t mask, int *sctx) {
    uint32_t *w = &c->T[l][2 * r + col];
    int gc = 2 * l + col;
    if (*w >> 31) return 0;
    if (c->passes == 3 && !any_sig_neighbour(c, r, gc)) {
        *w |= CPF;
        return 0;
    }
    lut_ptrs p = lut_at_plane(c->lvl[l], c->sb[l], b, c->levels);
    int ctx = sig_context(c, r, gc);
    uint32_t s = ac_decode(c, l, lut_get(c, p.sig + ctx));
    /* The encoder can only code a 1 here for b <= 27 (higher data bits are
     * flag bits that are 0 for coefficients in this pass). */
    if (s == 1 && (c->ref_quirk || b <= 27)) {
        *w |= mask;
        *w |= SIGMA;
        *sctx = sign_context(c, r, gc);
        return 1;
    }
    return 0;
}

/* CP_Decoder :546-589.  The reference decoder turns every decoded 1 into a
 * significant coefficient; the encoder does so only when the re-read data bit
 * is 1, which fails at b + 1 == 30 (the CP flag itself, :523-530) and at
 * b >= 28 in general.  ref_quirk selects the reference decoder's behaviour. */
static int cp_dec_sig(cbstate *c, int l, int r, int col, int b, uint32_t mask, int *sctx) {
    uint32_t *w = &c->T[l][2 * r + col];
    int gc = 2 * l + col;
    if (!((*w >> 30) & 1)) return 0;
    lut_ptrs p = lut_at_plane(c->lvl[l], c->sb[l], b, c->levels);
    int ctx = sig_context(c, r, gc);
    uint32_t s = ac_decode(c, l, lut_get(c, p.sig + p.cp_off + ctx));
    *w &= ~CPF;
    if (s == 1 && (c->ref_quirk || b <= 27)) {
        *w |= mask;
        *w |= SIGMA | REFF;
        *sctx = sign_context(c, r, gc);
        return 1;
    }
    return 0;
}

static void dec_sign(cbstate *c, int l, int r, int col, int b, int sctx, int cp) {
    uint32_t *w = &c->T[l][2 * r + col];
    lut_ptrs p = lut_at_plane(c->lvl[l], c->sb[l], b, c->levels);
    long base = p.sign + (cp ? p.cp_off : 0);
    uint32_t s = ac_decode(c, l, lut_get(c, base + (sctx >> 1)));
    s = ((s & 1) == (uint32_t)(sctx & 1)) ? 0u : 1u;
    *w |= s & 1;
}

/* MRP_Decoder :608-629 */
static void mrp_dec(cbstate *c, int l, int r, int col, int b, uint32_t mask, int P) {
    uint32_t *w = &c->T[l][2 * r + col];
    if ((*w >> 29) & 1) {
        uint32_t s = ac_decode(c, l, P);
        *w &= ~mask;
        *w |= mask & shl32((s << 1) + 1, b);
    } else if (*w >> 31)
        *w |= REFF;
}

static void dec_ctx_pass(cbstate *c, int b, uint32_t mask, int cp) {
    int pend[MAXL], sctx[MAXL];
    for (int r = 0; r < c->H; r++)
        for (int col = 0; col < 2; col++) {
            for (int l = 0; l < c->nl; l++)
                pend[l] = cp ? cp_dec_sig(c, l, r, col, b, mask, &sctx[l])
                             : spp_dec_sig(c, l, r, col, b, mask, &sctx[l]);
            for (int l = 0; l < c->nl; l++)
                if (pend[l]) dec_sign(c, l, r, col, b, sctx[l], cp);
        }
}

static void dec_mrp_pass(cbstate *c, int b, uint32_t mask) {
    for (int r = 0; r < c->H; r++)
        for (int col = 0; col < 2; col++)
            for (int l = 0; l < c->nl; l++) {
                lut_ptrs p = lut_at_plane(c->lvl[l], c->sb[l], b, c->levels);
                mrp_dec(c, l, r, col, b, mask, lut_get(c, p.ref));
            }
}

/* ------------------------------------------------------------------------- */
/* Codeblock drivers: kernels :1097-1224 + Encode/Decode :968-1090             */
/* ------------------------------------------------------------------------- */

typedef struct {
    int X, Y, passes, levels, cb;
    const int *lut;
    long lut_n;
    const int32_t *in;
    int32_t *out;
    int32_t *status; /* per codeblock, may be NULL */
    int ref_quirk;
    long ncb, next;
    const long *list; /* if not NULL: work item k is codeblock list[k] */
    pthread_mutex_t mu;
    int any_status;
    uint64_t *stats; /* LUT training counts (summed over the workers), or NULL */
    long stats_n;
} job;

static void setup_geometry(cbstate *c, const job *j, long k, int *x0, int *y0) {
    int ncbx = j->X / j->cb;
    c->passes = j->passes;
    c->levels = j->levels;
    c->H = j->cb;
    c->W = j->cb;
    c->nl = j->cb / 2;
    c->lut = j->lut;
    c->lut_n = j->lut_n;
    c->cap = (long)j->cb * j->cb;
    c->counter = 0;
    c->status = 0;
    c->ref_quirk = j->ref_quirk;
    *x0 = (int)(k % ncbx) * j->cb;
    *y0 = (int)(k / ncbx) * j->cb;
    for (int l = 0; l < c->nl; l++) {
        bpco_find_subband(*x0 + 2 * l, *y0, j->X, j->Y, j->levels, &c->lvl[l], &c->sb[l]);
        c->lower[l] = c->size[l] = c->resv[l] = c->cw[l] = 0;
        c->has_resv[l] = 0;
    }
}

static int encode_block(cbstate *c, const job *j, long k) {
    int x0, y0;
    setup_geometry(c, j, k, &x0, &y0);
    int32_t *slot = j->out + k * c->cap;
    c->stream = slot;
    for (long q = 0; q < c->cap; q++) slot[q] = -1; /* cudaMemset(out, -1) :1284 */
    /* Read_Coefficients :14-44 */
    uint32_t mx = 0;
    for (int l = 0; l < c->nl; l++)
        for (int r = 0; r < c->H; r++)
            for (int col = 0; col < 2; col++) {
                int32_t v = j->in[(long)(y0 + r) * j->X + x0 + 2 * l + col];
                uint32_t m = (uint32_t)(v < 0 ? -(int64_t)v : v);
                if (m >= (1u << 28)) c->status |= BPCO_ST_INPUT_RANGE;
                uint32_t w = (m << 1) + (v < 0 ? 1u : 0u);
                if (c->passes == 3) w |= CPF;
                c->T[l][2 * r + col] = w;
                mx |= w >> 1; /* Find_MSB :114-161 */
            }
    if (c->passes == 3) mx &= 0xDFFFFFFFu;
    int msb = 0;
    if (mx == 0)
        msb = 32;
    else {
        int hb = 31;
        while (!((mx >> hb) & 1)) hb--;
        msb = hb;
    }
    slot[0] = msb; /* :1155 */
    int b = msb;
    if (c->passes == 3) { /* :986-997 */
        enc_ctx_pass(c, b, 1);
        b--;
    }
    for (; b >= 0; b--) { /* :999-1018 */
        enc_ctx_pass(c, b, 0);
        enc_mrp_pass(c, b);
        if (c->passes == 3) enc_ctx_pass(c, b, 1);
    }
    for (int l = 0; l < c->nl; l++) { /* flush :1020 */
        if (!c->has_resv[l]) continue;
        if ((long)c->resv[l] < c->cap)
            slot[c->resv[l]] = (int32_t)c->lower[l];
        else
            c->status |= BPCO_ST_OVERFLOW;
    }
    return c->status;
}

static int decode_block(cbstate *c, const job *j, long k) {
    int x0, y0;
    setup_geometry(c, j, k, &x0, &y0);
    const int32_t *slot = j->in + k * c->cap;
    c->instr = slot;
    /* Initialize_Coefficients :65-81 */
    for (int l = 0; l < c->nl; l++)
        for (int q = 0; q < 2 * c->H; q++) c->T[l][q] = c->passes == 3 ? CPF : 0u;
    int msb = slot[0];
    /* an encoder writes 0..27 (|x| < 2^28) or 32 (all-zero codeblock) */
    if (msb < 0 || (msb > 27 && msb != 32)) {
        c->status |= BPCO_ST_BAD_STREAM;
        for (int l = 0; l < c->nl; l++)
            for (int q = 0; q < 2 * c->H; q++) c->T[l][q] = 0;
    } else {
        int b = msb;
        uint32_t mask = shl32(3u, b); /* :1038-1040 */
        if (b == 0) mask &= 2u;
        if (c->passes == 3) { /* :1045-1058 */
            dec_ctx_pass(c, b, mask, 1);
            b--;
            mask >>= 1;
            if (b == 0) mask = 2u;
        }
        for (; b >= 0; b--) { /* :1065-1088 */
            dec_ctx_pass(c, b, mask, 0);
            dec_mrp_pass(c, b, mask);
            if (c->passes == 3) dec_ctx_pass(c, b, mask, 1);
            mask >>= 1;
            if (b == 1) mask = 2u;
        }
    }
    /* Write_Coefficients :46-63 */
    for (int l = 0; l < c->nl; l++)
        for (int r = 0; r < c->H; r++)
            for (int col = 0; col < 2; col++) {
                uint32_t w = c->T[l][2 * r + col];
                int32_t v = (int32_t)((w & 0x1FFFFFFFu) >> 1);
                if (w & 1) v = -v;
                j->out[(long)(y0 + r) * j->X + x0 + 2 * l + col] = v;
            }
    return c->status;
}

typedef struct {
    job *j;
    int enc;
} worker_arg;

static void *worker(void *p) {
    worker_arg *a = (worker_arg *)p;
    job *j = a->j;
    cbstate *c = (cbstate *)malloc(sizeof(cbstate));
    c->stats = j->stats ? (uint64_t *)calloc((size_t)(2 * j->stats_n), sizeof(uint64_t)) : NULL;
    c->stats_n = j->stats_n;
    int st_all = 0;
    for (;;) {
        pthread_mutex_lock(&j->mu);
        long k = j->next;
        long chunk = 4;
        j->next += chunk;
        pthread_mutex_unlock(&j->mu);
        if (k >= j->ncb) break;
        long e = k + chunk < j->ncb ? k + chunk : j->ncb;
        for (; k < e; k++) {
            const long g = j->list ? j->list[k] : k;
            int st = a->enc ? encode_block(c, j, g) : decode_block(c, j, g);
            if (j->status) j->status[g] = st;
            st_all |= st;
        }
    }
    pthread_mutex_lock(&j->mu);
    j->any_status |= st_all;
    if (c->stats)
        for (long q = 0; q < 2 * j->stats_n; q++) j->stats[q] += c->stats[q];
    pthread_mutex_unlock(&j->mu);
    free(c->stats);
    free(c);
    return NULL;
}

static int run(int enc, const int32_t *in, int32_t *out, int X, int Y, const int *lut, int lut_n, int passes,
               int levels, int cb, int nthreads, int32_t *status, int ref_quirk, long cb_begin, long cb_end,
               uint64_t *stats, long stats_n, const long *list) {
    if (!in || !out || !lut || X <= 0 || Y <= 0 || (passes != 2 && passes != 3) || levels < 1 ||
        (cb != 64 && cb != 32) || X % cb || Y % cb)
        return BPCO_ERR_ARG;
    job j;
    memset(&j, 0, sizeof j);
    j.X = X;
    j.Y = Y;
    j.passes = passes;
    j.levels = levels;
    j.cb = cb;
    j.lut = lut;
    j.lut_n = lut_n;
    j.in = in;
    j.out = out;
    j.status = status;
    j.ref_quirk = ref_quirk;
    j.stats = stats;
    j.stats_n = stats_n;
    long ncb = (long)(X / cb) * (Y / cb);
    if (list) { /* cb_end = list length; every entry must name a codeblock */
        for (long k = 0; k < cb_end; k++)
            if (list[k] < 0 || list[k] >= ncb) return BPCO_ERR_ARG;
        ncb = cb_end;
        cb_begin = 0;
    }
    if (cb_end < 0 || cb_end > ncb) cb_end = ncb;
    if (cb_begin < 0) cb_begin = 0;
    j.ncb = cb_end;
    j.next = cb_begin;
    j.list = list;
    pthread_mutex_init(&j.mu, NULL);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    worker_arg wa = {&j, enc};
    for (int t = 0; t < nthreads; t++) pthread_create(&th[t], NULL, worker, &wa);
    for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
    pthread_mutex_destroy(&j.mu);
    return j.any_status;
}

/* Encode codeblocks [cb_begin, cb_end) of an X x Y raster (cb_end < 0: all).
 * out receives the slot stream (X*Y ints, codeblock-major slots of cb*cb ints).
 * Returns the OR of the per-codeblock status bits, or a negative error. */
int bpco_encode(const int32_t *img, int32_t *stream, int X, int Y, const int *lut, int lut_n, int passes, int levels,
                int cb, int nthreads, int32_t *status, long cb_begin, long cb_end) {
    return run(1, img, stream, X, Y, lut, lut_n, passes, levels, cb, nthreads, status, 0, cb_begin, cb_end, NULL, 0,
               NULL);
}

int bpco_decode(const int32_t *stream, int32_t *img, int X, int Y, const int *lut, int lut_n, int passes, int levels,
                int cb, int nthreads, int32_t *status, int ref_quirk, long cb_begin, long cb_end) {
    return run(0, stream, img, X, Y, lut, lut_n, passes, levels, cb, nthreads, status, ref_quirk, cb_begin,
               cb_end, NULL, 0, NULL);
}

/* bpco_encode / bpco_decode over the n codeblocks listed in `list` (indices in
 * raster order of codeblocks), for spot checks of images too large to code
 * whole; the slots and pixels of other codeblocks are left as they are. */
int bpco_encode_list(const int32_t *img, int32_t *stream, int X, int Y, const int *lut, int lut_n, int passes,
                     int levels, int cb, int nthreads, int32_t *status, const long *list, long n) {
    return run(1, img, stream, X, Y, lut, lut_n, passes, levels, cb, nthreads, status, 0, 0, n, NULL, 0, list);
}

int bpco_decode_list(const int32_t *stream, int32_t *img, int X, int Y, const int *lut, int lut_n, int passes,
                     int levels, int cb, int nthreads, int32_t *status, const long *list, long n) {
    return run(0, stream, img, X, Y, lut, lut_n, passes, levels, cb, nthreads, status, 0, 0, n, NULL, 0, list);
}

/* LUT training counts of an image: adds, for every entry of the LUT layout
 * with 15 planes (stats_n entries), stats[2k] += symbols coded with entry k
 * and stats[2k+1] += those equal to 1, over planes 0..14.  The encoder runs
 * with an all-64 table (the counts do not depend on the probabilities). */
int bpco_lut_stats(const int32_t *img, int X, int Y, int passes, int levels, int cb, int nthreads, uint64_t *stats,
                   long stats_n) {
    if (!stats || stats_n <= 0) return BPCO_ERR_ARG;
    int *lut = (int *)malloc(sizeof(int) * (size_t)stats_n);
    int32_t *scratch = (int32_t *)malloc(sizeof(int32_t) * (size_t)X * (size_t)Y);
    if (!lut || !scratch) {
        free(lut);
        free(scratch);
        return BPCO_ERR_ARG;
    }
    for (long q = 0; q < stats_n; q++) lut[q] = 64;
    int rc = run(1, img, scratch, X, Y, lut, (int)stats_n, passes, levels, cb, nthreads, NULL, 0, 0, -1, stats,
                 stats_n, NULL);
    free(lut);
    free(scratch);
    return rc < 0 ? rc : 0;
}

/* MSB of a codeblock as the kernel computes it (Find_MSB :114-161); for the
 * known-answer check against the sample image headers. */
int bpco_block_msb(const int32_t *img, int X, int x0, int y0, int cb, int passes) {
    uint32_t mx = 0;
    for (int r = 0; r < cb; r++)
        for (int q = 0; q < cb; q++) {
            int32_t v = img[(long)(y0 + r) * X + x0 + q];
            uint32_t m = (uint32_t)(v < 0 ? -(int64_t)v : v);
            uint32_t w = (m << 1) + (v < 0 ? 1u : 0u);
            if (passes == 3) w |= CPF;
            mx |= w >> 1;
        }
    if (passes == 3) mx &= 0xDFFFFFFFu;
    if (!mx) return 32;
    int hb = 31;
    while (!((mx >> hb) & 1)) hb--;
    return hb;
}
