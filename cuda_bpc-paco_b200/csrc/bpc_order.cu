// bpc_order.cu -- work order for images of several warp waves, and for the
// isolated decode of images of one or two waves.
//
// A CTA of the coder keeps its slot on the SM until its slowest warp is done,
// and the last wave of a launch runs on a partly idle GPU.  The time a warp
// spends on its codeblocks varies several-fold across an image (with the
// bitplanes coded and with how much the coder writes), so for images of many
// waves the coder is launched over the codeblocks sorted by expected work,
// heaviest first: warps of one CTA then get codeblocks of similar cost and
// the last wave holds the lightest ones.  The order changes only which warp
// codes which codeblock, never a stream word or a coefficient.
//
// Expected work of a work unit (the NG codeblocks one warp codes):
//   decoder: the slot words in use (MSB word + codewords), found by a binary
//            search for the first -1 of the fill (codewords are 0..0xFFFF;
//            on a damaged slot the search still ends inside it, and only the
//            order is affected), plus kPlaneWords per bitplane decoded;
//   encoder: the bitplanes coded, MSB + 1 (33 for an all-zero codeblock),
//            from one read of the coefficients.
// One CTA then counting-sorts the units by cost, descending (warp-aggregated
// shared-memory atomics; units of equal cost in any order).
//
// An isolated decode (launch_code) takes the first units of the order for its
// heavy launch and hands the rest out from a queue counter that follows the
// order and the keys in the scratch; the sorting CTA zeroes it.
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "bpc_kernels.h"

namespace bpc {

namespace {

constexpr int kBuckets = 1024;  // = threads of the sorting CTA
// decoder cost per plane in codeword-equivalents: a lockstep pass over a plane
// costs about as much as decoding 128 codewords (fit of per-codeblock decoder
// cycles on a B200 to words + planes).  For picking the few heaviest
// codeblocks of an isolated decode the planes weigh double: the chains that
// end last are those of the most planes (a 4096x4096 decode with 256: 0.560
// ms; with 128: 0.597 ms; with 64: 0.601 ms).
constexpr uint32_t kPlaneWords = 128, kPlaneWordsIso = 256;

template <int CBS>
__global__ void k_cost_dec(const int32_t *in, int ncb, uint32_t plane_words, uint32_t *key) {
    using G = Geo<CBS>;
    const int units = (ncb + G::NG - 1) / G::NG;
    for (int u = (int)(blockIdx.x * blockDim.x + threadIdx.x); u < units; u += (int)(gridDim.x * blockDim.x)) {
        uint32_t cost = 0;
        for (int k = 0; k < G::NG; k++) {
            const int cb = u * G::NG + k;
            if (cb >= ncb) break;
            const int32_t *slot = in + (size_t)cb * (size_t)G::CAP;
            int lo = 1, hi = G::CAP;  // first index >= 1 holding -1 (CAP if none)
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (__ldg(slot + mid) == -1)
                    hi = mid;
                else
                    lo = mid + 1;
            }
            const int m = __ldg(slot);  // MSB word: planes decoded
            const uint32_t planes = m == 32 ? 33u : (m >= 0 && m <= 27 ? (uint32_t)m + 1u : 0u);
            cost += (uint32_t)lo + plane_words * planes;
        }
        key[u] = cost;
    }
}

template <int CBS>
__global__ void k_cost_enc(const int32_t *in, int X, int ncbx, int ncb, uint32_t *key) {
    using G = Geo<CBS>;
    const int units = (ncb + G::NG - 1) / G::NG;
    const int lane = (int)(threadIdx.x & 31u), grp = lane / G::NL, gl = lane % G::NL;
    const int wstride = (int)(gridDim.x * blockDim.x) >> 5;
    for (int u = (int)(blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < units; u += wstride) {
        const int cb = u * G::NG + grp;
        uint32_t mx = 0;
        if (cb < ncb) {
            const int cbx = cb % ncbx, cby = cb / ncbx;
            const int32_t *src = in + (size_t)cby * CBS * (size_t)X + (size_t)cbx * CBS + 2 * gl;
            for (int i = 0; i < CBS; i++) {
                const int2 v = __ldg(reinterpret_cast<const int2 *>(src + (size_t)i * (size_t)X));
                mx |= (v.x < 0 ? 0u - (uint32_t)v.x : (uint32_t)v.x) | (v.y < 0 ? 0u - (uint32_t)v.y : (uint32_t)v.y);
            }
        }
        for (int o = G::NL / 2; o; o >>= 1) mx |= __shfl_xor_sync(0xffffffffu, mx, o);
        uint32_t cost = cb < ncb ? (mx ? 32u - (uint32_t)__clz((int)mx) : 33u) : 0u;
        if (G::NG == 2) cost += __shfl_xor_sync(0xffffffffu, cost, 16);
        if (lane == 0) key[u] = cost;
    }
}

// bin of a cost, descending: bin 0 holds the largest costs
__device__ __forceinline__ int cost_bin(uint32_t cost, int shift) {
    const uint32_t b = cost >> shift;
    return kBuckets - 1 - (int)(b > (uint32_t)(kBuckets - 1) ? (uint32_t)(kBuckets - 1) : b);
}

__global__ void __launch_bounds__(kBuckets) k_order(const uint32_t *key, int units, int shift, int ng, int *order,
                                                    int *ctr) {
    __shared__ uint32_t next[kBuckets];
    __shared__ uint32_t wsum[kBuckets / 32];
    const int tid = (int)threadIdx.x, lane = tid & 31;
    if (tid == 0 && ctr) *ctr = 0;  // the isolated decode's queue counter
    next[tid] = 0;
    __syncthreads();
    // whole warps step through the units together (full-mask warp calls)
    for (int u0 = tid - lane; u0 < units; u0 += kBuckets) {
        const int u = u0 + lane;
        const int bin = u < units ? cost_bin(key[u], shift) : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, bin);
        if (bin >= 0 && lane == __ffs(peers) - 1) atomicAdd(&next[bin], (uint32_t)__popc(peers));
    }
    __syncthreads();
    // exclusive scan of the bin counts
    const uint32_t v = next[tid];
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += t;
    }
    if (lane == 31) wsum[tid >> 5] = x;
    __syncthreads();
    if (tid < 32) {
        uint32_t y = wsum[tid];
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, y, o);
            if (lane >= o) y += t;
        }
        wsum[tid] = y;
    }
    __syncthreads();
    next[tid] = x - v + (tid >= 32 ? wsum[(tid >> 5) - 1] : 0u);
    __syncthreads();
    for (int u0 = tid - lane; u0 < units; u0 += kBuckets) {
        const int u = u0 + lane;
        const int bin = u < units ? cost_bin(key[u], shift) : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, bin);
        const int leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (bin >= 0 && lane == leader) base = atomicAdd(&next[bin], (uint32_t)__popc(peers));
        base = __shfl_sync(0xffffffffu, base, leader);
        const uint32_t rank = (uint32_t)__popc(peers & ((1u << lane) - 1u));
        if (bin >= 0) order[base + rank] = u * ng;
    }
}

}  // namespace

namespace {
// a device attribute, cached per device (callers may be on any host thread);
// 0 if it cannot be read
int cached_attr(cudaDeviceAttr a, std::atomic<int> *cache, int dev) {
    if (dev < 0 || dev >= 64) return 0;
    int n = cache[dev].load(std::memory_order_relaxed);
    if (!n) {
        if (cudaDeviceGetAttribute(&n, a, dev) != cudaSuccess || n <= 0) return 0;
        cache[dev].store(n, std::memory_order_relaxed);
    }
    return n;
}
}  // namespace

int sm_count(int dev) {
    static std::atomic<int> cache[64];
    return cached_attr(cudaDevAttrMultiProcessorCount, cache, dev);
}

int shared_optin(int dev) {
    static std::atomic<int> cache[64];
    return cached_attr(cudaDevAttrMaxSharedMemoryPerBlockOptin, cache, dev);
}

// warps resident at once on device `dev` (-1: the current device)
int resident_warps(bool enc, int dev) {
    if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return 1 << 30;
    const int n = sm_count(dev);
    if (n <= 0) return 1 << 30;
    return n * kWarps * (enc ? kMinCtasEnc : kMinCtasDec);
}

namespace {

template <int CBS>
cudaError_t plan_t(bool enc, Params &p, int *sched, cudaStream_t st, bool iso) {
    using G = Geo<CBS>;
    const int units = (p.ncb + G::NG - 1) / G::NG;
    uint32_t *key = reinterpret_cast<uint32_t *>(sched + units);
    const uint32_t plane_words = iso ? kPlaneWordsIso : kPlaneWords;
    if (enc) {  // one warp per unit, grid-stride
        const int grid = (units + 7) / 8 < 4096 ? (units + 7) / 8 : 4096;
        k_cost_enc<CBS><<<grid, 256, 0, st>>>(p.in, p.X, p.ncbx, p.ncb, key);
    } else {  // one thread per unit, grid-stride
        const int grid = (units + 255) / 256 < 1024 ? (units + 255) / 256 : 1024;
        k_cost_dec<CBS><<<grid, 256, 0, st>>>(p.in, p.ncb, plane_words, key);
    }
    // bins of 2^shift cost units: decoder costs reach NG * (CAP + 33 * plane
    // words), encoder costs 2 * 33
    int shift = 0;
    if (!enc) {
        const long long mx = (long long)G::NG * ((long long)G::CAP + 33LL * plane_words);
        while ((mx >> shift) > kBuckets - 1) shift++;
    }
    int *ctr = iso ? sched + 2 * units : nullptr;
    k_order<<<1, kBuckets, 0, st>>>(key, units, shift, G::NG, sched, ctr);
    p.order = sched;
    p.ctr = ctr;
    return cudaGetLastError();
}

}  // namespace

long long sched_ints(int ncb, int cbs) {
    const int ng = cbs == 64 ? 1 : 2;
    // order and cost keys, one int each per unit, then the queue counter
    return 2LL * ((ncb + ng - 1) / ng) + 4;
}

bool order_pays(bool enc, int ncb, int cbs, int dev) {
    const int ng = cbs == 64 ? 1 : 2;
    // an image within two waves gains nothing from a balanced last wave: every
    // unit starts at once or in the second wave anyway
    return (long long)((ncb + ng - 1) / ng) >= 2LL * resident_warps(enc, dev);
}

cudaError_t plan_order(bool enc, int cbs, Params &p, int *sched, cudaStream_t st, bool isolate) {
    p.order = nullptr;
    p.ctr = nullptr;
    if (!sched || p.offsets || p.cb_begin != 0 || p.cb_end != p.ncb) return cudaSuccess;
    if (order_pays(enc, p.ncb, cbs))
        return cbs == 64 ? plan_t<64>(enc, p, sched, st, false) : plan_t<32>(enc, p, sched, st, false);
    // isolated decode: 64x64 codeblocks, more than half a wave (smaller decodes
    // already spread one warp per CTA), more than the heavy launch's share, and
    // a device with SMs to spare for it
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return cudaSuccess;
    const long long res = resident_warps(false, dev);
    if (isolate && !enc && cbs == 64 && 2LL * p.ncb > res && p.ncb > 4 * kIsoCtas * kWarps &&
        sm_count(dev) > 4 * kIsoCtas && shared_optin(dev) > 0)
        return plan_t<64>(enc, p, sched, st, true);
    return cudaSuccess;
}

}  // namespace bpc
