// bpc_dwt.cu -- reversible CDF 5/3 lifting DWT (JPEG 2000 integer filter) on
// the GPU, in the Mallat layout the coder's subband finder assumes: after each
// level the top-left (H >> l) x (W >> l) region holds [L | H] along x and
// [L ; H] along y.  Input and output are int32 rasters (the caller applies any
// DC level shift).  Symmetric extension: x[n] = x[n-2] for the predict step,
// d[-1] = d[0] for the update step; floor division by arithmetic shifts.
//
//   predict:  d[i] = x[2i+1] - floor((x[2i] + x[2i+2]) / 2)
//   update:   s[i] = x[2i]   + floor((d[i-1] + d[i] + 2) / 4)
//
// Rows: one CTA per row, the row staged in shared memory.  Columns: one thread
// per (row pair, column), so every access is coalesced along the row; predict
// and update are two kernels through a scratch raster the caller provides.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>

#include "../../include/bpc_paco.h"

namespace {

__global__ void k_rows_fwd(int32_t *data, long long stride, int w, int h) {
    extern __shared__ int32_t sm[];
    int32_t *x = sm, *d = sm + w;
    const int half = w >> 1;
    for (int r = blockIdx.x; r < h; r += gridDim.x) {
        int32_t *p = data + (long long)r * stride;
        for (int k = threadIdx.x; k < w; k += blockDim.x) x[k] = p[k];
        __syncthreads();
        for (int i = threadIdx.x; i < half; i += blockDim.x) {
            const int32_t a = x[2 * i], b = (2 * i + 2 < w) ? x[2 * i + 2] : x[w - 2];
            d[i] = x[2 * i + 1] - ((a + b) >> 1);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < half; i += blockDim.x) {
            const int32_t dm = i ? d[i - 1] : d[0];
            p[i] = x[2 * i] + ((dm + d[i] + 2) >> 2);
            p[half + i] = d[i];
        }
        __syncthreads();
    }
}

__global__ void k_rows_inv(int32_t *data, long long stride, int w, int h) {
    extern __shared__ int32_t sm[];
    int32_t *s = sm, *d = sm + (w >> 1), *e = sm + w;  // e: even samples
    const int half = w >> 1;
    for (int r = blockIdx.x; r < h; r += gridDim.x) {
        int32_t *p = data + (long long)r * stride;
        for (int k = threadIdx.x; k < w; k += blockDim.x) sm[k] = p[k];
        __syncthreads();
        for (int i = threadIdx.x; i < half; i += blockDim.x) {
            const int32_t dm = i ? d[i - 1] : d[0];
            e[i] = s[i] - ((dm + d[i] + 2) >> 2);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < half; i += blockDim.x) {
            const int32_t en = (i + 1 < half) ? e[i + 1] : e[half - 1];
            p[2 * i] = e[i];
            p[2 * i + 1] = d[i] + ((e[i] + en) >> 1);
        }
        __syncthreads();
    }
}

// columns, forward: predict into tmp rows [h/2, h), then update into tmp rows [0, h/2)
__global__ void k_cols_predict(const int32_t *x, int32_t *tmp, long long stride, int w, int h) {
    const int half = h >> 1;
    const long long n = (long long)half * w;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / w), c = (int)(t % w);
        const int32_t a = x[(long long)(2 * i) * stride + c];
        const int32_t b = x[(long long)(2 * i + 2 < h ? 2 * i + 2 : h - 2) * stride + c];
        tmp[(long long)(half + i) * stride + c] = x[(long long)(2 * i + 1) * stride + c] - ((a + b) >> 1);
    }
}
__global__ void k_cols_update(const int32_t *x, int32_t *tmp, long long stride, int w, int h) {
    const int half = h >> 1;
    const long long n = (long long)half * w;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / w), c = (int)(t % w);
        const int32_t d = tmp[(long long)(half + i) * stride + c];
        const int32_t dm = tmp[(long long)(half + (i ? i - 1 : 0)) * stride + c];
        tmp[(long long)i * stride + c] = x[(long long)(2 * i) * stride + c] + ((dm + d + 2) >> 2);
    }
}
// columns, inverse: undo update into tmp even rows, then predict into tmp odd rows
__global__ void k_cols_unupdate(const int32_t *x, int32_t *tmp, long long stride, int w, int h) {
    const int half = h >> 1;
    const long long n = (long long)half * w;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / w), c = (int)(t % w);
        const int32_t d = x[(long long)(half + i) * stride + c];
        const int32_t dm = x[(long long)(half + (i ? i - 1 : 0)) * stride + c];
        tmp[(long long)(2 * i) * stride + c] = x[(long long)i * stride + c] - ((dm + d + 2) >> 2);
    }
}
__global__ void k_cols_unpredict(const int32_t *x, int32_t *tmp, long long stride, int w, int h) {
    const int half = h >> 1;
    const long long n = (long long)half * w;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / w), c = (int)(t % w);
        const int32_t e0 = tmp[(long long)(2 * i) * stride + c];
        const int32_t e1 = tmp[(long long)(2 * i + 2 < h ? 2 * i + 2 : h - 2) * stride + c];
        tmp[(long long)(2 * i + 1) * stride + c] = x[(long long)(half + i) * stride + c] + ((e0 + e1) >> 1);
    }
}
__global__ void k_copy_region(const int32_t *src, int32_t *dst, long long stride, int w, int h) {
    const long long n = (long long)h * w;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long r = t / w, c = t % w;
        dst[r * stride + c] = src[r * stride + c];
    }
}

int grid_for(long long n) { return (int)((n + 255) / 256 < 148 * 32 ? (n + 255) / 256 : 148 * 32); }

int check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        std::fprintf(stderr, "bpc dwt: %s: %s\n", what, cudaGetErrorString(e));
        return BPC_ERR_CUDA;
    }
    return BPC_OK;
}

bool valid(const int *d, const int *t, int X, int Y, int levels) {
    if (!d || !t || X <= 0 || Y <= 0 || levels < 0 || levels > 16) return false;
    // every level halves an even extent of at least 2
    return (X % (2 << (levels ? levels - 1 : 0))) == 0 && (Y % (2 << (levels ? levels - 1 : 0))) == 0 &&
           (X >> (levels ? levels - 1 : 0)) >= 2 && (Y >> (levels ? levels - 1 : 0)) >= 2 && X <= 32768;
}

}  // namespace

extern "C" {

int bpc_dwt53_forward(int *d_data, int X, int Y, int levels, int *d_tmp, void *stream) {
    if (!valid(d_data, d_tmp, X, Y, levels)) return BPC_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t sm = (size_t)(X + X / 2) * sizeof(int32_t);
    int rc = check(cudaFuncSetAttribute(k_rows_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm), "attr");
    if (rc) return rc;
    for (int l = 0; l < levels; l++) {
        const int w = X >> l, h = Y >> l;
        k_rows_fwd<<<h < 148 * 8 ? h : 148 * 8, 256, (size_t)(w + w / 2) * 4, st>>>(d_data, X, w, h);
        const long long n = (long long)(h / 2) * w;
        k_cols_predict<<<grid_for(n), 256, 0, st>>>(d_data, d_tmp, X, w, h);
        k_cols_update<<<grid_for(n), 256, 0, st>>>(d_data, d_tmp, X, w, h);
        k_copy_region<<<grid_for((long long)w * h), 256, 0, st>>>(d_tmp, d_data, X, w, h);
        if ((rc = check(cudaGetLastError(), "launch"))) return rc;
    }
    return BPC_OK;
}

int bpc_dwt53_inverse(int *d_data, int X, int Y, int levels, int *d_tmp, void *stream) {
    if (!valid(d_data, d_tmp, X, Y, levels)) return BPC_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t sm = (size_t)(X + X / 2) * sizeof(int32_t);
    int rc = check(cudaFuncSetAttribute(k_rows_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm), "attr");
    if (rc) return rc;
    for (int l = levels - 1; l >= 0; l--) {
        const int w = X >> l, h = Y >> l;
        const long long n = (long long)(h / 2) * w;
        k_cols_unupdate<<<grid_for(n), 256, 0, st>>>(d_data, d_tmp, X, w, h);
        k_cols_unpredict<<<grid_for(n), 256, 0, st>>>(d_data, d_tmp, X, w, h);
        k_copy_region<<<grid_for((long long)w * h), 256, 0, st>>>(d_tmp, d_data, X, w, h);
        k_rows_inv<<<h < 148 * 8 ? h : 148 * 8, 256, (size_t)(w + w / 2) * 4, st>>>(d_data, X, w, h);
        if ((rc = check(cudaGetLastError(), "launch"))) return rc;
    }
    return BPC_OK;
}

}  // extern "C"
