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
// Per level, forward: the row step reads the level's region from the data
// raster and writes it to a scratch raster the caller provides, the column
// step reads it back and writes the data raster (the inverse runs columns, then
// rows).  Each step is one kernel in which a thread lifts a run of pairs of one
// row (16-byte loads and stores) or one column (a warp covers 32 adjacent
// columns, so every access is coalesced).
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>

#include "../../include/bpc_paco.h"

namespace {

// All four kernels work out of place (data -> scratch -> data per level), so
// each level reads and writes its region exactly once per direction of the
// row step and once for the column step.  A thread computes K consecutive
// lifting pairs of one row (or column) from its own inputs plus a two-sample
// halo on the left and one on the right; neighbouring threads read the halo
// samples again, from L1.

// forward, along a row: in[0, w) -> out[0, w/2) = s, out[w/2, w) = d
template <int K>
__global__ void k_rows_fwd(const int32_t *in, int32_t *out, long long stride, int w, int h) {
    const int half = w >> 1;
    const int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * K;
    const int r = blockIdx.y;
    if (i0 >= half || r >= h) return;
    const int32_t *p = in + (long long)r * stride;
    int32_t *q = out + (long long)r * stride;
    int32_t x[2 * K + 1];
    const bool vec = 2 * i0 + 2 * K < w && (((uintptr_t)(p + 2 * i0)) & 15) == 0 && K % 2 == 0;
    if (vec) {
#pragma unroll
        for (int k = 0; k < 2 * K; k += 4) {
            const int4 v = *reinterpret_cast<const int4 *>(p + 2 * i0 + k);
            x[k] = v.x;
            x[k + 1] = v.y;
            x[k + 2] = v.z;
            x[k + 3] = v.w;
        }
        x[2 * K] = p[2 * i0 + 2 * K];
    } else {
#pragma unroll
        for (int k = 0; k <= 2 * K; k++) {
            const int e = 2 * i0 + k;
            x[k] = p[e < w ? e : w - 2];  // x[w] = x[w - 2]; samples past it are never used
        }
    }
    int32_t dprev = 0;
    if (i0 > 0) dprev = p[2 * i0 - 1] - ((p[2 * i0 - 2] + x[0]) >> 1);
    int32_t sv[K], dv[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
        const int i = i0 + k;
        const int32_t xn = 2 * i + 2 < w ? x[2 * k + 2] : x[2 * k];  // x[w] = x[w - 2]
        const int32_t d = x[2 * k + 1] - ((x[2 * k] + xn) >> 1);
        const int32_t dm = i == 0 ? d : dprev;
        sv[k] = x[2 * k] + ((dm + d + 2) >> 2);
        dv[k] = d;
        dprev = d;
    }
    if (i0 + K <= half && (((uintptr_t)(q + i0)) & 15) == 0 && (((uintptr_t)(q + half + i0)) & 15) == 0 &&
        K % 4 == 0) {
#pragma unroll
        for (int k = 0; k < K; k += 4) {
            *reinterpret_cast<int4 *>(q + i0 + k) = make_int4(sv[k], sv[k + 1], sv[k + 2], sv[k + 3]);
            *reinterpret_cast<int4 *>(q + half + i0 + k) = make_int4(dv[k], dv[k + 1], dv[k + 2], dv[k + 3]);
        }
    } else {
#pragma unroll
        for (int k = 0; k < K; k++)
            if (i0 + k < half) {
                q[i0 + k] = sv[k];
                q[half + i0 + k] = dv[k];
            }
    }
}

// V adjacent columns per thread, loaded and stored together (V = 4: 16-byte
// accesses, a warp covers 128 columns of a row)
template <int V>
struct Cols {
    int32_t v[V];
};
template <int V>
__device__ __forceinline__ Cols<V> ld(const int32_t *p) {
    Cols<V> r;
    if constexpr (V == 4) {
        const int4 t = *reinterpret_cast<const int4 *>(p);
        r.v[0] = t.x, r.v[1] = t.y, r.v[2] = t.z, r.v[3] = t.w;
    } else {
#pragma unroll
        for (int k = 0; k < V; k++) r.v[k] = p[k];
    }
    return r;
}
template <int V>
__device__ __forceinline__ void st(int32_t *p, const Cols<V> &r) {
    if constexpr (V == 4) {
        *reinterpret_cast<int4 *>(p) = make_int4(r.v[0], r.v[1], r.v[2], r.v[3]);
    } else {
#pragma unroll
        for (int k = 0; k < V; k++) p[k] = r.v[k];
    }
}

// forward, along a column: rows [0, h) -> rows [0, h/2) = s, [h/2, h) = d
template <int K, int V>
__global__ void k_cols_fwd(const int32_t *in, int32_t *out, long long stride, int w, int h) {
    const int c = (blockIdx.x * blockDim.x + threadIdx.x) * V;
    const int half = h >> 1;
    const int i0 = blockIdx.y * K;
    if (c >= w || i0 >= half) return;
    auto X = [&](int row) { return ld<V>(in + (long long)(row < h ? row : h - 2) * stride + c); };
    Cols<V> dprev{}, xe = X(2 * i0);
    if (i0 > 0) {
        const Cols<V> a = X(2 * i0 - 2), b = X(2 * i0 - 1);
#pragma unroll
        for (int k = 0; k < V; k++) dprev.v[k] = b.v[k] - ((a.v[k] + xe.v[k]) >> 1);
    }
#pragma unroll
    for (int k = 0; k < K; k++) {
        const int i = i0 + k;
        if (i >= half) break;
        const Cols<V> xn = X(2 * i + 2), xo = X(2 * i + 1);  // x[h] = x[h - 2]
        Cols<V> sv, dv;
#pragma unroll
        for (int u = 0; u < V; u++) {
            const int32_t d = xo.v[u] - ((xe.v[u] + xn.v[u]) >> 1);
            const int32_t dm = i == 0 ? d : dprev.v[u];
            sv.v[u] = xe.v[u] + ((dm + d + 2) >> 2);
            dv.v[u] = d;
        }
        st<V>(out + (long long)i * stride + c, sv);
        st<V>(out + (long long)(half + i) * stride + c, dv);
        dprev = dv;
        xe = xn;
    }
}

// inverse, along a column: rows [0, h/2) = s, [h/2, h) = d -> rows [0, h)
template <int K, int V>
__global__ void k_cols_inv(const int32_t *in, int32_t *out, long long stride, int w, int h) {
    const int c = (blockIdx.x * blockDim.x + threadIdx.x) * V;
    const int half = h >> 1;
    const int i0 = blockIdx.y * K;
    if (c >= w || i0 >= half) return;
    auto S = [&](int i) { return ld<V>(in + (long long)i * stride + c); };
    auto D = [&](int i) { return ld<V>(in + (long long)(half + i) * stride + c); };
    Cols<V> di = D(i0), e, s0 = S(i0), dm = i0 ? D(i0 - 1) : di;
#pragma unroll
    for (int u = 0; u < V; u++) e.v[u] = s0.v[u] - ((dm.v[u] + di.v[u] + 2) >> 2);
#pragma unroll
    for (int k = 0; k < K; k++) {
        const int i = i0 + k;
        if (i >= half) break;
        Cols<V> en = e, dn = di;
        if (i + 1 < half) {  // x[h] = x[h - 2] at the end
            dn = D(i + 1);
            const Cols<V> sn = S(i + 1);
#pragma unroll
            for (int u = 0; u < V; u++) en.v[u] = sn.v[u] - ((di.v[u] + dn.v[u] + 2) >> 2);
        }
        Cols<V> odd;
#pragma unroll
        for (int u = 0; u < V; u++) odd.v[u] = di.v[u] + ((e.v[u] + en.v[u]) >> 1);
        st<V>(out + (long long)(2 * i) * stride + c, e);
        st<V>(out + (long long)(2 * i + 1) * stride + c, odd);
        e = en;
        di = dn;
    }
}

// inverse, along a row: [0, w/2) = s, [w/2, w) = d -> [0, w)
template <int K>
__global__ void k_rows_inv(const int32_t *in, int32_t *out, long long stride, int w, int h) {
    const int half = w >> 1;
    const int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * K;
    const int r = blockIdx.y;
    if (i0 >= half || r >= h) return;
    const int32_t *p = in + (long long)r * stride;
    int32_t *q = out + (long long)r * stride;
    int32_t di = p[half + i0];
    int32_t e = p[i0] - (((i0 ? p[half + i0 - 1] : di) + di + 2) >> 2);
    int32_t xv[2 * K];
#pragma unroll
    for (int k = 0; k < K; k++) {
        const int i = i0 + k;
        int32_t en = e, dn = di;
        if (i + 1 < half) {
            dn = p[half + i + 1];
            en = p[i + 1] - ((di + dn + 2) >> 2);
        }
        xv[2 * k] = e;
        xv[2 * k + 1] = di + ((e + en) >> 1);
        e = en;
        di = dn;
    }
    if (2 * i0 + 2 * K <= w && (((uintptr_t)(q + 2 * i0)) & 15) == 0 && K % 2 == 0) {
#pragma unroll
        for (int k = 0; k < 2 * K; k += 4)
            *reinterpret_cast<int4 *>(q + 2 * i0 + k) = make_int4(xv[k], xv[k + 1], xv[k + 2], xv[k + 3]);
    } else {
#pragma unroll
        for (int k = 0; k < 2 * K; k++)
            if (2 * i0 + k < w) q[2 * i0 + k] = xv[k];
    }
}

// 16-byte column accesses: both rasters 16-byte aligned, row stride and level
// width multiples of 4 ints
bool vec4(const int *a, const int *b, int stride, int w) {
    return ((((uintptr_t)a) | ((uintptr_t)b)) & 15) == 0 && stride % 4 == 0 && w % 4 == 0;
}

constexpr int kRowPairs = 4;   // lifting pairs per thread along a row
constexpr int kColPairs = 8;   // ... along a column
constexpr int kThreads = 128;

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
           (X >> (levels ? levels - 1 : 0)) >= 2 && (Y >> (levels ? levels - 1 : 0)) >= 2 && X <= 32768 && Y <= 65535;
}

}  // namespace

extern "C" {

int bpc_dwt53_forward(int *d_data, int X, int Y, int levels, int *d_tmp, void *stream) {
    if (!valid(d_data, d_tmp, X, Y, levels)) return BPC_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    for (int l = 0; l < levels; l++) {
        const int w = X >> l, h = Y >> l;
        const dim3 gr((unsigned)((w / 2 + kThreads * kRowPairs - 1) / (kThreads * kRowPairs)), (unsigned)h);
        k_rows_fwd<kRowPairs><<<gr, kThreads, 0, st>>>(d_data, d_tmp, X, w, h);
        if (vec4(d_data, d_tmp, X, w)) {
            const dim3 gc((unsigned)((w / 4 + kThreads - 1) / kThreads), (unsigned)((h / 2 + kColPairs - 1) / kColPairs));
            k_cols_fwd<kColPairs, 4><<<gc, kThreads, 0, st>>>(d_tmp, d_data, X, w, h);
        } else {
            const dim3 gc((unsigned)((w + kThreads - 1) / kThreads), (unsigned)((h / 2 + kColPairs - 1) / kColPairs));
            k_cols_fwd<kColPairs, 1><<<gc, kThreads, 0, st>>>(d_tmp, d_data, X, w, h);
        }
        const int rc = check(cudaGetLastError(), "launch");
        if (rc) return rc;
    }
    return BPC_OK;
}

int bpc_dwt53_inverse(int *d_data, int X, int Y, int levels, int *d_tmp, void *stream) {
    if (!valid(d_data, d_tmp, X, Y, levels)) return BPC_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    for (int l = levels - 1; l >= 0; l--) {
        const int w = X >> l, h = Y >> l;
        if (vec4(d_data, d_tmp, X, w)) {
            const dim3 gc((unsigned)((w / 4 + kThreads - 1) / kThreads), (unsigned)((h / 2 + kColPairs - 1) / kColPairs));
            k_cols_inv<kColPairs, 4><<<gc, kThreads, 0, st>>>(d_data, d_tmp, X, w, h);
        } else {
            const dim3 gc((unsigned)((w + kThreads - 1) / kThreads), (unsigned)((h / 2 + kColPairs - 1) / kColPairs));
            k_cols_inv<kColPairs, 1><<<gc, kThreads, 0, st>>>(d_data, d_tmp, X, w, h);
        }
        const dim3 gr((unsigned)((w / 2 + kThreads * kRowPairs - 1) / (kThreads * kRowPairs)), (unsigned)h);
        k_rows_inv<kRowPairs><<<gr, kThreads, 0, st>>>(d_tmp, d_data, X, w, h);
        const int rc = check(cudaGetLastError(), "launch");
        if (rc) return rc;
    }
    return BPC_OK;
}

}  // extern "C"
