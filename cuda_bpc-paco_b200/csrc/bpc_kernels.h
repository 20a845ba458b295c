// bpc_kernels.h -- launcher interface between the C ABI (bpc_api.cu) and the
// sm_100a kernels (bpc_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include "bpc_core.cuh"

#ifndef ENC_MIN_CTAS
#define ENC_MIN_CTAS 4
#endif

namespace bpc {

constexpr int kWarps = 4;  // warps (codeblocks) per CTA
// CTAs per SM the register budget is sized for: the decoder steps its lanes
// together and needs many warps to hide latency (7 x 4 warps, <= 72
// registers); the encoder runs each lane's coder on its own and needs the
// registers more than the warps.
#ifndef DEC_MIN_CTAS
#define DEC_MIN_CTAS 7
#endif
constexpr int kMinCtasDec = DEC_MIN_CTAS;
constexpr int kMinCtasEnc = ENC_MIN_CTAS;

// Input alignment the kernels' vector loads need: the encoder reads each
// lane's two coefficients with one 8-byte load, the decoder reads the slot
// stream with 16-byte loads.  Entry points refuse other pointers (a misaligned
// vector load would fault and lose the CUDA context).
constexpr unsigned kEncInAlign = 8, kDecInAlign = 16;
inline bool aligned_to(const void *p, unsigned a) { return ((uintptr_t)p & (uintptr_t)(a - 1)) == 0; }

// Launch the encoder (enc) or decoder over p.ncb codeblocks.  grid <= 0 picks
// one CTA per kWarps codeblocks; a positive grid runs persistent CTAs that
// walk the codeblocks grid-stride.  latency_forms lets a launch of a few waves
// take the latency forms of the coder loops (and one-warp CTAs for a small
// decode), which finish a launch alone on the GPU sooner but execute more
// instructions; callers that run many launches at once pass false.
cudaError_t launch_code(bool enc, int passes, int cbs, const Params &p, int grid, cudaStream_t st,
                        bool latency_forms = true);

// One plain (sched null) or work-ordered launch over codeblocks
// [cb_begin, cb_end) (cb_end < 0: all) after the C ABI's argument checks
// (bpc_api.cu); returns a BPC_* code.
int code_device(bool enc, const int *in, int *out, int X, int Y, const int *d_lut, int lut_n, int passes, int levels,
                int cb, int *d_status, int *d_counts, int grid, void *stream, int cb_begin = 0, int cb_end = -1,
                int *sched = nullptr, bool latency_forms = true);

// Work order for a whole-image launch (bpc_order.cu): with scratch `sched` of
// sched_ints(ncb, cbs) ints, queue the kernels that sort the image's work
// units by expected cost, heaviest first, and set p.order.  Images of more than
// two waves are sorted for a balanced last wave; decodes of 64x64 codeblocks
// between half a wave and two waves are sorted for an isolated launch
// (launch_code) when `isolate` allows it, which also sets p.ctr to the bulk
// launch's queue counter in the scratch.  Other images keep raster order
// (p.order and p.ctr stay null).
long long sched_ints(int ncb, int cbs);
// SMs of device `dev`, and its opt-in shared memory per block (cached)
int sm_count(int dev);
int shared_optin(int dev);
// warps of the plain coder resident at once on device `dev` (-1: current)
int resident_warps(bool enc, int dev);
// more than two waves on device `dev` (-1: the current device)
bool order_pays(bool enc, int ncb, int cbs, int dev = -1);
cudaError_t plan_order(bool enc, int cbs, Params &p, int *sched, cudaStream_t st, bool isolate);
// heavy CTAs of an isolated decode (kWarps codeblocks each)
constexpr int kIsoCtas = 6;

// LUT training: add, per LUT entry, [2k] symbols coded and [2k+1] symbols
// equal to 1 over p.ncb codeblocks of p.in (planes 0..14) to stats.
cudaError_t launch_stats(int passes, int cbs, const Params &p, unsigned long long *stats, cudaStream_t st);

}  // namespace bpc
