// bpc_kernels.cu -- sm_100a kernels of the BPC-PaCo coder and their launcher.
//
// One warp codes one 64x64 codeblock (or two 32x32 codeblocks); a CTA of
// kWarps warps stages the LUT once into shared memory as bytes and then walks
// codeblocks grid-stride, so the same kernel serves the plain one-image launch
// (grid = ceil(ncb / kWarps)) and a persistent launch (grid = k * 148).
// The decoder's kMinCtasDec CTAs per SM (28 warps) keep every codeblock of a
// 4096x4096 image resident in one wave.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "bpc_core.cuh"
#include "bpc_kernels.h"

namespace bpc {

struct GpuWarp {
    __device__ __forceinline__ int lane() const { return (int)(threadIdx.x & 31u); }
    __device__ __forceinline__ uint32_t ballot(bool p) { return __ballot_sync(0xffffffffu, p); }
    __device__ __forceinline__ bool any(bool p) { return __any_sync(0xffffffffu, p) != 0; }
    __device__ __forceinline__ uint32_t reduce_or(uint32_t v) { return __reduce_or_sync(0xffffffffu, v); }
    __device__ __forceinline__ uint32_t shfl_xor(uint32_t v, int o) { return __shfl_xor_sync(0xffffffffu, v, o); }
    __device__ __forceinline__ uint32_t shfl_up(uint32_t v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }
    __device__ __forceinline__ uint32_t shfl_down(uint32_t v, int d) { return __shfl_down_sync(0xffffffffu, v, d); }
    __device__ __forceinline__ uint32_t shfl_idx(uint32_t v, int l) { return __shfl_sync(0xffffffffu, v, l); }
    __device__ __forceinline__ void smem_or(uint32_t *p, uint32_t v) { atomicOr(p, v); }
    __device__ __forceinline__ void sync() { __syncwarp(); }
    __device__ __forceinline__ void syncmask(uint32_t m) { __syncwarp(m); }
    __device__ __forceinline__ void load2(const int32_t *p, int32_t &a, int32_t &b) {
        const int2 v = __ldg(reinterpret_cast<const int2 *>(p));
        a = v.x;
        b = v.y;
    }
    __device__ __forceinline__ int32_t load1(const int32_t *p) { return __ldg(p); }
    __device__ __forceinline__ void store1(int32_t *p, int32_t a) { *p = a; }
    __device__ __forceinline__ void store2(int32_t *p, int32_t a, int32_t b) {
        *reinterpret_cast<int2 *>(p) = make_int2(a, b);
    }
    __device__ __forceinline__ void load4(const int32_t *p, uint32_t &a, uint32_t &b, uint32_t &c, uint32_t &d) {
        const int4 v = __ldg(reinterpret_cast<const int4 *>(p));
        a = (uint32_t)v.x;
        b = (uint32_t)v.y;
        c = (uint32_t)v.z;
        d = (uint32_t)v.w;
    }
    __device__ __forceinline__ void atomic_or(int *p, int v) { atomicOr(p, v); }
};

// WARPS codeblock warps per CTA: kWarps, or 1 for decodes of at most half a wave
// (their heaviest codeblocks then land on different SMs, see launch_t); the
// register budget stays that of kMinCtas x kWarps resident warps per SM
template <int PASSES, int CBS, bool ENC, int WARPS = kWarps, int LAT = 0>
__global__ void __launch_bounds__(WARPS * 32, (ENC ? kMinCtasEnc : kMinCtasDec) * kWarps / WARPS) k_bpc(Params p) {
    using G = Geo<CBS>;
    const int heavy = ENC ? 0 : p.heavy;
    // heavy launch of an isolated decode: the bulk launch (its programmatic
    // dependent) may start as soon as every heavy CTA has reached this point
    if (heavy == 1) asm volatile("griddepcontrol.launch_dependents;");
    extern __shared__ __align__(16) unsigned char smem[];
    uint8_t *tab = smem;
    int bad = 0;
    for (int k = (int)threadIdx.x; k < p.tab_n; k += (int)blockDim.x) {
        int v = k < p.lut_n ? __ldg(p.lut + k) : 0;
        if (v < 0 || v > 255) {
            bad = 1;
            v = 0;
        }
        tab[k] = (uint8_t)v;
    }
    if (bad && p.status) atomicOr(p.status, ST_LUT_RANGE);
    uint8_t *sgtab = smem + p.tab_n;
    if (!ENC) build_sign_table(sgtab, (int)threadIdx.x, (int)blockDim.x);
    __syncthreads();
    const int warp = (int)(threadIdx.x >> 5);
    // per warp: the decoder's codeword ring, or the encoder's event ranking words
    uint32_t *ring =
        reinterpret_cast<uint32_t *>(smem + p.tab_n + kSignTableBytes) + warp * (ENC ? 512 : G::RING_WORDS);
    GpuWarp w;
    uint32_t planes[28][4];  // per-thread bitplanes (local memory, L1-resident)
    uint8_t ev_key[ENC ? kEvKeys : 1];
    uint32_t ev_val[ENC ? kEvVals : 1];
    // Walk: heavy 0, codeblocks cb_begin + slot*NG, grid-stride; heavy 1, the
    // order's unit `slot` if slot < heavy_n; heavy 2, the order's unit
    // heavy_n + slot, then the units past every warp slot's first one, each
    // taken by the first warp to come back for work.
    const int slot = (int)blockIdx.x * WARPS + warp, nslots = (int)gridDim.x * WARPS;
    const int units = (p.ncb + G::NG - 1) / G::NG;
    int pos = heavy == 1 ? (slot < p.heavy_n ? slot : p.heavy_n)
                         : (heavy == 2 ? p.heavy_n + slot : p.cb_begin + slot * G::NG);
    const int lim = heavy == 1 ? p.heavy_n : (heavy == 2 ? units : p.cb_end);
    while (pos < lim) {
        {
            Coder<PASSES, CBS, ENC, GpuWarp, LAT> cd(w, p, ring, tab, sgtab, planes, ev_key, ev_val);
            cd.run(heavy ? p.order[pos] : (p.order ? p.order[pos / G::NG] : pos));
        }
        if (heavy == 1) {
            pos = lim;
        } else if (heavy == 2) {
            int nx = 0;
            if ((threadIdx.x & 31u) == 0u) nx = atomicAdd(p.ctr, 1);
            pos = p.heavy_n + nslots + __shfl_sync(0xffffffffu, nx, 0);
        } else {
            pos += nslots * G::NG;
        }
    }
    // bulk launch of an isolated decode: it completes only after the heavy
    // launch, its programmatic prerequisite, has completed and its stores are
    // visible, so whatever follows in the stream sees both
    if (heavy == 2) asm volatile("griddepcontrol.wait;" ::: "memory");
}

// LUT training counts: the encoder's pass masks without its arithmetic coder
template <int PASSES, int CBS>
__global__ void __launch_bounds__(kWarps * 32, kMinCtasEnc) k_bpc_stats(Params p, unsigned long long *stats) {
    using G = Geo<CBS>;
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = (int)(threadIdx.x >> 5);
    uint32_t *ring = reinterpret_cast<uint32_t *>(smem) + warp * 512;
    GpuWarp w;
    uint32_t planes[28][4];
    uint8_t ev_key[1];
    uint32_t ev_val[1];
    const int stride = (int)gridDim.x * kWarps * G::NG;
    for (int base = p.cb_begin + ((int)blockIdx.x * kWarps + warp) * G::NG; base < p.cb_end; base += stride) {
        Coder<PASSES, CBS, true, GpuWarp> cd(w, p, ring, nullptr, nullptr, planes, ev_key, ev_val);
        cd.template run<true>(base, stats);
    }
}

template <int PASSES, int CBS>
static cudaError_t launch_stats_t(const Params &p, unsigned long long *stats, cudaStream_t st) {
    using G = Geo<CBS>;
    const size_t sm = (size_t)kWarps * 4u * 512u;
    const int warps_needed = (p.cb_end - p.cb_begin + G::NG - 1) / G::NG;
    const int grid = (warps_needed + kWarps - 1) / kWarps;
    if (grid < 1) return cudaSuccess;
    k_bpc_stats<PASSES, CBS><<<grid, kWarps * 32, sm, st>>>(p, stats);
    return cudaGetLastError();
}

cudaError_t launch_stats(int passes, int cbs, const Params &p, unsigned long long *stats, cudaStream_t st) {
    if (p.cb_end <= p.cb_begin) return cudaSuccess;
    if (passes == 2) return cbs == 64 ? launch_stats_t<2, 64>(p, stats, st) : launch_stats_t<2, 32>(p, stats, st);
    return cbs == 64 ? launch_stats_t<3, 64>(p, stats, st) : launch_stats_t<3, 32>(p, stats, st);
}

template <int PASSES, int CBS, bool ENC, int WARPS>
static size_t smem_bytes(const Params &p) {
    using G = Geo<CBS>;
    return (size_t)p.tab_n + (size_t)kSignTableBytes + (size_t)WARPS * 4u * (size_t)(ENC ? 512 : G::RING_WORDS);
}

// The shared memory a launch asks for grows with the LUT's length, and the
// attribute that admits it belongs to the kernel, not to the launch: host
// threads set it and launch under this lock, so no launch meets a smaller
// setting another thread made in between.
static std::mutex &attr_mu() {
    static std::mutex m;
    return m;
}

template <int PASSES, int CBS, bool ENC, int WARPS, int LAT>
static cudaError_t launch_w(const Params &p, int grid, int warps_needed, cudaStream_t st) {
    std::lock_guard<std::mutex> lk(attr_mu());
    const size_t sm = smem_bytes<PASSES, CBS, ENC, WARPS>(p);
    cudaError_t e = cudaFuncSetAttribute(k_bpc<PASSES, CBS, ENC, WARPS, LAT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    const int full = (warps_needed + WARPS - 1) / WARPS;
    if (grid <= 0 || grid > full) grid = full;
    if (grid < 1) grid = 1;
    k_bpc<PASSES, CBS, ENC, WARPS, LAT><<<grid, WARPS * 32, sm, st>>>(p);
    return cudaGetLastError();
}

// Isolated decode of a work-ordered image of one or two waves (p.order and
// p.ctr from plan_order).  Its heaviest kIsoCtas x kWarps codeblocks run
// first, in CTAs that take their SM's whole shared memory, so no other CTA
// shares their SMs and each of their warps has a sub-partition to itself
// (latency form of the step).  The rest of the image is a programmatic
// dependent launch: it starts once every heavy CTA is resident, fills the other
// SMs, one codeblock per warp slot, and the codeblocks beyond its warp slots go
// to whichever warps finish first.  In a one-wave decode the heaviest
// codeblocks' chains otherwise run beside 27 other warps and set the launch
// time (4096x4096, 3-pass: 0.62 -> 0.54 ms).
template <int PASSES, int CBS>
static cudaError_t launch_iso(const Params &p, cudaStream_t st) {
    using G = Geo<CBS>;
    std::lock_guard<std::mutex> lk(attr_mu());
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const int optin = shared_optin(dev), sms = sm_count(dev);
    if (optin <= 0 || sms <= kIsoCtas) return cudaErrorInvalidValue;
    const int units = (p.ncb + G::NG - 1) / G::NG;
    Params ph = p;
    ph.heavy = 1;
    ph.heavy_n = kIsoCtas * kWarps;
    e = cudaFuncSetAttribute(k_bpc<PASSES, CBS, false, kWarps, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             optin);
    if (e != cudaSuccess) return e;
    k_bpc<PASSES, CBS, false, kWarps, 1><<<kIsoCtas, kWarps * 32, (size_t)optin, st>>>(ph);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    Params pb = ph;
    pb.heavy = 2;
    const size_t sm = smem_bytes<PASSES, CBS, false, kWarps>(pb);
    e = cudaFuncSetAttribute(k_bpc<PASSES, CBS, false, kWarps, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sm);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bpc<PASSES, CBS, false, kWarps, 0>, kWarps * 32,
                                                      sm);
    if (e != cudaSuccess) return e;
    const int full = (units - ph.heavy_n + kWarps - 1) / kWarps;
    int grid = (sms - kIsoCtas) * (per_sm > 0 ? per_sm : 1);
    if (grid > full) grid = full;
    if (grid < 1) grid = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kWarps * 32);
    cfg.dynamicSmemBytes = sm;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, k_bpc<PASSES, CBS, false, kWarps, 0>, pb);
    if (e == cudaErrorNotSupported) {
        // no programmatic launch here: the bulk then runs after the heavy
        // launch in plain stream order (its final wait returns at once)
        (void)cudaGetLastError();
        cfg.numAttrs = 0;
        e = cudaLaunchKernelEx(&cfg, k_bpc<PASSES, CBS, false, kWarps, 0>, pb);
    }
    return e;
}

template <int PASSES, int CBS, bool ENC>
static cudaError_t launch_t(const Params &p, int grid, cudaStream_t st, bool lat) {
    using G = Geo<CBS>;
    const int warps_needed = (p.cb_end - p.cb_begin + G::NG - 1) / G::NG;
    const long long resident = resident_warps(ENC, -1);
    if constexpr (ENC) {
        // Encodes of at most two waves end with the serial chains of their
        // heaviest codeblocks: the latency forms of the symbol loop, three
        // positions per iteration within one wave (a 2048x2048 encode: 0.180
        // -> 0.154 ms), two within two waves (4096x4096: 0.417 -> 0.412 ms;
        // three there: 0.430).  Longer encodes are issue-bound and keep the
        // form with fewer instructions.
        if (lat && grid <= 0 && warps_needed <= resident)
            return launch_w<PASSES, CBS, ENC, kWarps, 2>(p, grid, warps_needed, st);
        if (lat && grid <= 0 && warps_needed <= 2 * resident)
            return launch_w<PASSES, CBS, ENC, kWarps, 1>(p, grid, warps_needed, st);
        return launch_w<PASSES, CBS, ENC, kWarps, 0>(p, grid, warps_needed, st);
    } else {
        // A decode of at most half a wave of resident warps runs one warp per
        // CTA (consecutive CTAs go to different SMs, so its heaviest codeblocks,
        // the coarse subbands, neighbours in raster order, do not share an SM's
        // instruction cache and shared-memory pipes; a 2048x2048 decode: 0.375
        // -> 0.358 ms) and the latency form of the step.  Fuller decodes keep
        // 4-warp CTAs and the form with fewer instructions, which measured
        // faster there.  A work-ordered whole image the planner marked for
        // isolation (p.ctr set) runs its heaviest codeblocks on SMs of their own.
        if constexpr (CBS == 64) {
            if (lat && grid <= 0 && p.order && p.ctr) return launch_iso<PASSES, CBS>(p, st);
        }
        if (lat && grid <= 0 && 2LL * warps_needed <= resident)
            return launch_w<PASSES, CBS, ENC, 1, 1>(p, grid, warps_needed, st);
        return launch_w<PASSES, CBS, ENC, kWarps, 0>(p, grid, warps_needed, st);
    }
}

cudaError_t launch_code(bool enc, int passes, int cbs, const Params &p, int grid, cudaStream_t st, bool lat) {
    if (p.cb_end <= p.cb_begin) return cudaSuccess;
    if (enc) {
        if (passes == 2)
            return cbs == 64 ? launch_t<2, 64, true>(p, grid, st, lat) : launch_t<2, 32, true>(p, grid, st, lat);
        return cbs == 64 ? launch_t<3, 64, true>(p, grid, st, lat) : launch_t<3, 32, true>(p, grid, st, lat);
    }
    if (passes == 2)
        return cbs == 64 ? launch_t<2, 64, false>(p, grid, st, lat) : launch_t<2, 32, false>(p, grid, st, lat);
    return cbs == 64 ? launch_t<3, 64, false>(p, grid, st, lat) : launch_t<3, 32, false>(p, grid, st, lat);
}

}  // namespace bpc
