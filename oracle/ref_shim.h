/* ref_shim.h -- forced-include shim that lets the reference kernel source
 * (source/BPC_PaCo.cu, written for pre-Volta GPUs) compile for sm_100a.
 *
 * TEST INFRASTRUCTURE ONLY (builds the secondary oracle in oracle/_ref/).
 * The reference calls the legacy warp intrinsics __shfl, __shfl_up,
 * __shfl_down (BPC_PaCo.cu:142-148, :357-383) and __ballot (:270, :306), which
 * do not exist for compute_70+.  They are mapped to their _sync forms:
 * shuffles over the full warp (every call site is reached by all 32 lanes) and
 * the ballot over the lanes active at the call (__activemask), the closest
 * sm_70+ equivalent of the pre-Volta "lanes that reached this call" meaning.
 */
#pragma once
#define __shfl_down(v, d) __shfl_down_sync(0xffffffffu, (v), (d))
#define __shfl_up(v, d) __shfl_up_sync(0xffffffffu, (v), (d))
#define __shfl(v, l) __shfl_sync(0xffffffffu, (v), (l))
#define __ballot(p) __ballot_sync(__activemask(), (p))
