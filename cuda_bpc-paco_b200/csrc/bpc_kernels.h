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

// Launch the encoder (enc) or decoder over p.ncb codeblocks.  grid <= 0 picks
// one CTA per kWarps codeblocks; a positive grid runs persistent CTAs that
// walk the codeblocks grid-stride.
cudaError_t launch_code(bool enc, int passes, int cbs, const Params &p, int grid, cudaStream_t st);

// LUT training: add, per LUT entry, [2k] symbols coded and [2k+1] symbols
// equal to 1 over p.ncb codeblocks of p.in (planes 0..14) to stats.
cudaError_t launch_stats(int passes, int cbs, const Params &p, unsigned long long *stats, cudaStream_t st);

}  // namespace bpc
