// bpc_noalloc.cu -- a one-image encode into the compact container that
// allocates no device memory.
//
// Who needs it.  Some callers cannot call cudaMalloc while they code an image:
// a host application that has already handed its device memory budget to a
// pool it manages itself, a latency-critical pipeline that must not let an
// allocation synchronise the device in the middle of its stream, or a plugin
// that its host framework only ever gives device pointers.  Producing the
// compact container needs scratch beyond the caller's input and outputs (the
// slot stream the encoder writes, the per-codeblock codeword counts and
// container sizes, and the prefix-scan workspace); bpc_batch_encode gets it
// from the batch object, which allocates.  This entry point instead keeps all
// of that scratch in one fixed-size array declared at file scope below, so the
// caller passes only the input, the outputs and a stream.
//
// Cost and limits.  The array is kScratchBytes (16.1 MiB); every GPU on which
// this library's code for it is loaded holds it until the process exits.  An
// image may have at most kMaxWords coefficients (2048 x 2048); larger ones are
// rejected with BPC_ERR_TOO_LARGE before anything runs.
//
// Sharing.  Every call uses the same array and the array keeps the last
// call's contents.  Nothing in it has to start at zero: the encoder writes
// every word of each slot and every codeword count, and the sizes are written
// in full before the scan reads them.  Calls whose work overlaps on the GPU
// (two streams, two host threads) race on the array and corrupt each other's
// results; serialise them.
//
// Set-up.  Host code only knows the array by a host-side stand-in name, not by
// its device address; passing the name to a kernel would fault or, where the
// GPU can reach host memory, silently use the wrong memory.  So the first call
// on each device (with that device current) looks the device address up with
// cudaGetSymbolAddress and keeps it, together with the CUDA context it belongs
// to; make that first call before any stream capture begins.  A kept address
// is only valid in its context: after cudaDeviceReset (or any other change of
// the device's current context) the next call sees a different context and
// looks the address up again, which makes that call a set-up call too.
#include <cuda.h>  // CUcontext; cuCtxGetCurrent itself comes from the runtime's entry-point query
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <cub/device/device_scan.cuh>
#include <mutex>

#include "../../include/bpc_paco.h"
#include "bpc_core.cuh"
#include "bpc_kernels.h"

namespace {

constexpr long long kMaxWords = 2048LL * 2048LL;    // coefficients per image
constexpr long long kMaxCb = kMaxWords / (32 * 32);  // codeblocks (32x32 worst case)
constexpr size_t kSlotBytes = (size_t)kMaxWords * 4;
constexpr size_t kCountBytes = (size_t)kMaxCb * 4;
constexpr size_t kSizeBytes = (size_t)kMaxCb * 8;
constexpr size_t kScanBytes = 64 * 1024;
constexpr size_t kScratchBytes = kSlotBytes + kCountBytes + kSizeBytes + kScanBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char *g_addr[kMaxDevices] = {};
CUcontext g_ctx[kMaxDevices] = {};

// the calling thread's current CUDA context (null if none yet, or if the
// driver entry point cannot be found)
CUcontext current_context() {
    using Fn = CUresult (*)(CUcontext *);
    static const Fn fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return (Fn)f;
    }();
    CUcontext c = nullptr;
    if (!fn || fn(&c) != CUDA_SUCCESS) return nullptr;
    return c;
}

// container words per codeblock: MSB + codewords, capped at the slot size
__global__ void k_noalloc_sizes(const int *counts, long long ncb, long long cap, long long *sizes) {
    for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < ncb;
         g += (long long)gridDim.x * blockDim.x) {
        const long long n = (long long)counts[g] + 1;
        sizes[g] = n < cap ? n : cap;
    }
}

// one warp per codeblock copies its slot's first words into the container
__global__ void k_noalloc_gather(const int32_t *slots, long long cap, const long long *offsets, long long ncb,
                                 int32_t *compact) {
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long g = warp; g < ncb; g += nw) {
        const long long o0 = offsets[g], n = offsets[g + 1] - o0;
        for (long long q = lane; q < n; q += 32) compact[o0 + q] = slots[g * cap + q];
    }
}

// device address of the array on the current device (looked up once per
// device and context)
int scratch_address(unsigned char **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) return BPC_ERR_CUDA;
    std::lock_guard<std::mutex> g(g_mu);
    const CUcontext ctx = current_context();
    if (!g_addr[dev] || !ctx || ctx != g_ctx[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            std::fprintf(stderr, "bpc: cudaGetSymbolAddress(scratch) failed: %s\n", cudaGetErrorString(e));
            return BPC_ERR_CUDA;
        }
        size_t need = 0;
        e = cub::DeviceScan::InclusiveSum(nullptr, need, (const long long *)nullptr, (long long *)nullptr, (int)kMaxCb);
        if (e != cudaSuccess || need > kScanBytes) {
            std::fprintf(stderr, "bpc: prefix-scan workspace (%zu bytes) does not fit the fixed scratch\n", need);
            return BPC_ERR_CUDA;
        }
        g_addr[dev] = (unsigned char *)p;
        g_ctx[dev] = current_context();  // the lookup made the device's context current
    }
    *out = g_addr[dev];
    return BPC_OK;
}

}  // namespace

extern "C" int bpc_encode_compact_noalloc(const int *d_coeffs, int X, int Y, const int *d_lut, int lut_n, int passes,
                                          int levels, int cb_size, int *d_compact, long long *d_offsets,
                                          int *d_status, void *stream) {
    if (!d_coeffs || !d_lut || lut_n <= 0 || !d_compact || !d_offsets || (passes != 2 && passes != 3) ||
        (cb_size != 64 && cb_size != 32) || levels < 1 || levels > 16 || X <= 0 || Y <= 0 || X % cb_size ||
        Y % cb_size || !bpc::aligned_to(d_coeffs, bpc::kEncInAlign))
        return BPC_ERR_ARG;
    if ((long long)X * (long long)Y > kMaxWords) {
        std::fprintf(stderr, "bpc: %d x %d exceeds the %lld coefficients of the no-allocation entry point\n", X, Y,
                     kMaxWords);
        return BPC_ERR_TOO_LARGE;
    }
    unsigned char *base = nullptr;
    int rc = scratch_address(&base);
    if (rc) return rc;
    int32_t *slots = (int32_t *)base;
    int *counts = (int *)(base + kSlotBytes);
    long long *sizes = (long long *)(base + kSlotBytes + kCountBytes);
    void *scan_tmp = base + kSlotBytes + kCountBytes + kSizeBytes;
    cudaStream_t st = (cudaStream_t)stream;

    // the plain encoder, writing its slot stream and counts into the array
    bpc::Params p;
    const bpc::LutOffsets o = bpc::lut_offsets(levels, passes, lut_n);
    p.in = d_coeffs;
    p.out = slots;
    p.lut = d_lut;
    p.lut_n = lut_n;
    p.tab_n = o.tab_n;
    p.X = X;
    p.Y = Y;
    p.levels = levels;
    p.ncbx = X / cb_size;
    p.ncb = (X / cb_size) * (Y / cb_size);
    p.a_sig = o.a_sig;
    p.a_sign = o.a_sign;
    p.cp_off = o.cp_off;
    p.status = d_status;
    p.counts = counts;
    p.offsets = nullptr;
    p.cb_begin = 0;
    p.cb_end = p.ncb;
    cudaError_t e = bpc::launch_code(true, passes, cb_size, p, 0, st);
    const long long ncb = p.ncb, cap = (long long)cb_size * cb_size;
    if (e == cudaSuccess) {
        k_noalloc_sizes<<<(int)((ncb + 255) / 256), 256, 0, st>>>(counts, ncb, cap, sizes);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(d_offsets, 0, sizeof(long long), st);
    if (e == cudaSuccess) {
        size_t tmp = kScanBytes;
        e = cub::DeviceScan::InclusiveSum(scan_tmp, tmp, sizes, d_offsets + 1, (int)ncb, st);
    }
    if (e == cudaSuccess) {
        const int blocks = (int)((ncb * 32 + 255) / 256);
        k_noalloc_gather<<<blocks, 256, 0, st>>>(slots, cap, d_offsets, ncb, d_compact);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        std::fprintf(stderr, "bpc: no-allocation encode failed: %s\n", cudaGetErrorString(e));
        return BPC_ERR_CUDA;
    }
    return BPC_OK;
}
