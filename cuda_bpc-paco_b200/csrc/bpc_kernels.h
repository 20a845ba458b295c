// bpc_kernels.h -- launcher interface between the C ABI (bpc_api.cu) and the
// sm_100a kernels (bpc_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include "bpc_core.cuh"

namespace bpc {

constexpr int kWarps = 4;    // warps (codeblocks) per CTA
constexpr int kMinCtas = 7;  // CTAs per SM the register budget is sized for

// Launch the encoder (enc) or decoder over p.ncb codeblocks.  grid <= 0 picks
// one CTA per kWarps codeblocks; a positive grid runs persistent CTAs that
// walk the codeblocks grid-stride.
cudaError_t launch_code(bool enc, int passes, int cbs, const Params &p, int grid, cudaStream_t st);

}  // namespace bpc
