// emu_warp.cpp -- the coder's device code (cuda_bpc-paco_b200/csrc/bpc_core.cuh)
// compiled for the host and run one codeblock warp at a time, each of the 32
// lanes on its own user-level context (ucontext), every warp collective a
// barrier of the lanes that take part in it.  TEST ONLY: it lets the CPU test
// suite run the product's bitstream logic -- the exact source the kernels are
// built from -- against the oracle without a GPU.  It is never part of the
// product library.
#include <ucontext.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "bpc_core.cuh"

namespace {

constexpr int kStack = 512 * 1024;

// Cooperative scheduler of the 32 lane contexts of one warp.  Barrier kinds:
// 0 = all lanes, 1 / 2 = lanes 0-15 / 16-31 (the two 16-lane groups of 32x32
// codeblocks).  A lane waiting at a barrier runs again only once every lane of
// that barrier has arrived.
struct Sched {
    ucontext_t main_ctx;
    ucontext_t ctx[32];
    std::vector<char> stack[32];
    bool done[32];
    int waitk[32];
    unsigned waitgen[32];
    unsigned gen[3];
    int cnt[3];
    int cur;
    uint32_t slot[32];
};
Sched *S = nullptr;

void barrier(int k) {
    static const int need[3] = {32, 16, 16};
    const int l = S->cur;
    S->waitk[l] = k;
    S->waitgen[l] = S->gen[k];
    if (++S->cnt[k] == need[k]) {
        S->cnt[k] = 0;
        S->gen[k]++;
    }
    swapcontext(&S->ctx[l], &S->main_ctx);
}

struct EmuWarp {
    int id;
    int lane() const { return id; }
    template <class F>
    uint32_t exch(uint32_t v, F f) {  // deposit, meet, read everyone's, meet again
        S->slot[id] = v;
        barrier(0);
        const uint32_t r = f(S->slot);
        barrier(0);
        return r;
    }
    uint32_t ballot(bool p) {
        return exch(p ? 1u : 0u, [](const uint32_t *s) {
            uint32_t m = 0;
            for (int k = 0; k < 32; k++) m |= (s[k] & 1u) << k;
            return m;
        });
    }
    bool any(bool p) { return ballot(p) != 0; }
    uint32_t reduce_or(uint32_t v) {
        return exch(v, [](const uint32_t *s) {
            uint32_t m = 0;
            for (int k = 0; k < 32; k++) m |= s[k];
            return m;
        });
    }
    uint32_t shfl_xor(uint32_t v, int o) {
        const int src = (id ^ o) & 31;
        return exch(v, [src](const uint32_t *s) { return s[src]; });
    }
    uint32_t shfl_up(uint32_t v, int d) {  // lanes below d keep their own value
        const int src = id - d >= 0 ? id - d : id;
        return exch(v, [src](const uint32_t *s) { return s[src]; });
    }
    uint32_t shfl_down(uint32_t v, int d) {
        const int src = id + d < 32 ? id + d : id;
        return exch(v, [src](const uint32_t *s) { return s[src]; });
    }
    uint32_t shfl_idx(uint32_t v, int l) {
        const int src = l & 31;
        return exch(v, [src](const uint32_t *s) { return s[src]; });
    }
    void smem_or(uint32_t *p, uint32_t v) { *p |= v; }
    void sync() { barrier(0); }
    void syncmask(uint32_t m) { barrier(m == 0xffffffffu ? 0 : (m == 0x0000ffffu ? 1 : 2)); }
    void load2(const int32_t *p, int32_t &a, int32_t &b) { a = p[0], b = p[1]; }
    int32_t load1(const int32_t *p) { return *p; }
    void store1(int32_t *p, int32_t a) { *p = a; }
    void store2(int32_t *p, int32_t a, int32_t b) { p[0] = a, p[1] = b; }
    void load4(const int32_t *p, uint32_t &a, uint32_t &b, uint32_t &c, uint32_t &d) {
        a = (uint32_t)p[0], b = (uint32_t)p[1], c = (uint32_t)p[2], d = (uint32_t)p[3];
    }
    void atomic_or(int *p, int v) { *p |= v; }
};

struct Job {
    const bpc::Params *p;
    const uint8_t *tab, *sgtab;
    uint32_t *ring;
    int base;
    unsigned long long *stats;
    int kind;  // 0 code, 1 statistics, 2 / 3 code with the latency forms of the loops (LAT 1 / 2)
};
Job *J = nullptr;

template <int PASSES, int CBS, bool ENC>
void lane_main() {
    const int l = S->cur;
    EmuWarp w{l};
    uint32_t planes[28][4];
    uint8_t ev_key[ENC ? bpc::kEvKeys : 1];
    uint32_t ev_val[ENC ? bpc::kEvVals : 1];
    if (J->kind == 2) {  // the latency forms of the loops
        bpc::Coder<PASSES, CBS, ENC, EmuWarp, 1> cd(w, *J->p, J->ring, J->tab, J->sgtab, planes, ev_key, ev_val);
        cd.run(J->base);
        S->done[l] = true;
        return;
    }
    if (J->kind == 3) {
        bpc::Coder<PASSES, CBS, ENC, EmuWarp, 2> cd(w, *J->p, J->ring, J->tab, J->sgtab, planes, ev_key, ev_val);
        cd.run(J->base);
        S->done[l] = true;
        return;
    }
    bpc::Coder<PASSES, CBS, ENC, EmuWarp> cd(w, *J->p, J->ring, J->tab, J->sgtab, planes, ev_key, ev_val);
    if constexpr (ENC) {
        if (J->kind == 1)
            cd.template run<true>(J->base, J->stats);
        else
            cd.run(J->base);
    } else {
        cd.run(J->base);
    }
    S->done[l] = true;
}

template <int PASSES, int CBS, bool ENC>
int run_warp(Job &job) {
    J = &job;
    for (int l = 0; l < 32; l++) {
        S->done[l] = false;
        S->waitk[l] = -1;
        getcontext(&S->ctx[l]);
        S->ctx[l].uc_stack.ss_sp = S->stack[l].data();
        S->ctx[l].uc_stack.ss_size = kStack;
        S->ctx[l].uc_link = &S->main_ctx;
        makecontext(&S->ctx[l], (void (*)())lane_main<PASSES, CBS, ENC>, 0);
    }
    for (int k = 0; k < 3; k++) S->gen[k] = 0, S->cnt[k] = 0;
    for (;;) {
        bool all = true, progress = false;
        for (int l = 0; l < 32; l++) {
            if (S->done[l]) continue;
            all = false;
            const int k = S->waitk[l];
            if (k >= 0 && S->gen[k] == S->waitgen[l]) continue;  // barrier not complete yet
            S->waitk[l] = -1;
            S->cur = l;
            swapcontext(&S->main_ctx, &S->ctx[l]);
            progress = true;
        }
        if (all) return 0;
        if (!progress) return -1;  // lanes wait at different barriers: divergent collective
    }
}

template <int PASSES, int CBS, bool ENC>
int run_all(const bpc::Params &p, const uint8_t *tab, const uint8_t *sgtab, unsigned long long *stats, int kind) {
    using G = bpc::Geo<CBS>;
    std::vector<uint32_t> ring(ENC ? 512 : G::RING_WORDS, 0u);
    for (int base = p.cb_begin; base < p.cb_end; base += G::NG) {
        Job job{&p, tab, sgtab, ring.data(), base, stats, kind};
        if (run_warp<PASSES, CBS, ENC>(job)) return -1;
    }
    return 0;
}

}  // namespace

// enc = 1 encode (kind 0: slot stream, kind 1: LUT statistics into stats,
// kind 2 / 3: slot stream with the latency forms of the loops), enc = 0 decode (of
// the slot stream, or of the compact container when offsets is not null; kind
// 2: with the latency form).  Returns the OR of the status bits, or -1 if the lanes of a
// warp ever met different collectives.
extern "C" int emu_code(int enc, int kind, int passes, int cbs, const int32_t *in, int32_t *out, int X, int Y,
                        const int32_t *lut, int lut_n, int levels, unsigned long long *stats,
                        const long long *offsets) {
    Sched sched;
    for (int l = 0; l < 32; l++) sched.stack[l].assign(kStack, 0);
    S = &sched;
    const bpc::LutOffsets o = bpc::lut_offsets(levels, passes, lut_n);
    std::vector<uint8_t> tab((size_t)o.tab_n, 0), sg(bpc::kSignTableBytes, 0);
    int status = 0;
    for (int k = 0; k < o.tab_n; k++) {
        int v = k < lut_n ? lut[k] : 0;
        if (v < 0 || v > 255) status |= bpc::ST_LUT_RANGE, v = 0;
        tab[k] = (uint8_t)v;
    }
    bpc::build_sign_table(sg.data(), 0, 1);
    bpc::Params p;
    p.in = in;
    p.out = out;
    p.lut = lut;
    p.lut_n = lut_n;
    p.tab_n = o.tab_n;
    p.X = X;
    p.Y = Y;
    p.levels = levels;
    p.ncbx = X / cbs;
    p.ncb = (X / cbs) * (Y / cbs);
    p.a_sig = o.a_sig;
    p.a_sign = o.a_sign;
    p.cp_off = o.cp_off;
    p.status = &status;
    p.counts = nullptr;
    p.offsets = enc ? nullptr : offsets;  // decode from the compact container when given
    p.in_words = (long long)X * Y;       // the container lies in the X*Y-word input buffer
    p.cb_begin = 0;
    p.cb_end = p.ncb;
    int rc;
    const uint8_t *t = tab.data(), *g = sg.data();
    if (enc) {
        if (passes == 2)
            rc = cbs == 64 ? run_all<2, 64, true>(p, t, g, stats, kind) : run_all<2, 32, true>(p, t, g, stats, kind);
        else
            rc = cbs == 64 ? run_all<3, 64, true>(p, t, g, stats, kind) : run_all<3, 32, true>(p, t, g, stats, kind);
    } else {
        if (passes == 2)
            rc = cbs == 64 ? run_all<2, 64, false>(p, t, g, stats, kind) : run_all<2, 32, false>(p, t, g, stats, kind);
        else
            rc = cbs == 64 ? run_all<3, 64, false>(p, t, g, stats, kind) : run_all<3, 32, false>(p, t, g, stats, kind);
    }
    S = nullptr;
    return rc ? rc : status;
}
