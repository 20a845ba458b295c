// bpc_api.cu -- C ABI of the codec (declared in include/bpc_paco.h).
//
// The drop-in pair CUDA_BPC / load_LUTs keeps the reference's buffer contract
// (source/BPC_PaCo.cu:1277-1325, source/main_example.cu:219-448); the
// status-returning and device-pointer variants expose the same kernels with an
// explicit mode, LUT length and stream.  There is no CPU path: every coding
// call launches the sm_100a kernels of bpc_kernels.cu.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <map>
#include <mutex>
#include <vector>

#include "../../include/bpc_paco.h"
#include "bpc_core.cuh"
#include "bpc_kernels.h"
#include "bpc_lut.h"

namespace {

struct DropInState {
    std::mutex mu;
    int passes = 2, levels = 5, cb = 64;
    int last = 0;
    std::map<const int *, int> lut_len;  // device LUTs handed out by load_LUTs
    // device buffers reused across CUDA_BPC calls (grow only)
    int *d_a = nullptr, *d_b = nullptr, *d_status = nullptr;
    size_t cap = 0;
    // host-buffer calls run bands of codeblock rows round-robin on `nstreams`
    // of these streams so that the copies in both directions overlap the
    // kernels; a band holds at least `band_cbs` codeblocks and there are at
    // most `max_bands` of them (bpc_set_host_pipeline)
    static constexpr int kMaxStreams = 16;
    int band_cbs = 512, max_bands = 32, nstreams = 16, ramp = 3;
    cudaStream_t streams[kMaxStreams] = {};
    cudaEvent_t done[kMaxStreams] = {};
};

DropInState &state() {
    static DropInState s;
    return s;
}

bool valid_mode(int passes, int levels, int cb) {
    return (passes == 2 || passes == 3) && levels >= 1 && levels <= 16 && (cb == 64 || cb == 32);
}

bool valid_geometry(int X, int Y, int cb, int levels) {
    if (X <= 0 || Y <= 0 || X % cb || Y % cb) return false;
    if ((long long)X * (long long)Y > (1LL << 31) - 1) return false;
    (void)levels;
    return true;
}

int fill_params(bpc::Params &p, bool enc, const int *in, int *out, int X, int Y, const int *d_lut, int lut_n,
                int passes, int levels, int cb, int *d_status, int *d_counts) {
    if (!valid_mode(passes, levels, cb) || !valid_geometry(X, Y, cb, levels) || !in || !out || !d_lut || lut_n <= 0)
        return BPC_ERR_ARG;
    if (!bpc::aligned_to(in, enc ? bpc::kEncInAlign : bpc::kDecInAlign)) return BPC_ERR_ARG;
    const bpc::LutOffsets o = bpc::lut_offsets(levels, passes, lut_n);
    p.in = in;
    p.out = out;
    p.lut = d_lut;
    p.lut_n = lut_n;
    p.tab_n = o.tab_n;
    p.X = X;
    p.Y = Y;
    p.levels = levels;
    p.ncbx = X / cb;
    p.ncb = (X / cb) * (Y / cb);
    p.a_sig = o.a_sig;
    p.a_sign = o.a_sign;
    p.cp_off = o.cp_off;
    p.status = d_status;
    p.counts = d_counts;
    p.offsets = nullptr;
    p.cb_begin = 0;
    p.cb_end = p.ncb;
    return BPC_OK;
}


#define CUDA_TRY(x)                                                                              \
    do {                                                                                         \
        cudaError_t e_ = (x);                                                                    \
        if (e_ != cudaSuccess) {                                                                 \
            std::fprintf(stderr, "bpc: %s failed: %s\n", #x, cudaGetErrorString(e_));            \
            return BPC_ERR_CUDA;                                                                 \
        }                                                                                        \
    } while (0)

// Bands of codeblock rows for the host-buffer pipeline, as the row where each
// band starts plus `rows` at the end.  The input rows and the output slots of
// a band are contiguous in both layouts (coefficients row-major, slots in
// raster order of codeblocks).  Bands hold at least band_cbs codeblocks (each
// band's kernel still spreads over the SMs) and there are at most max_bands of
// the steady length (shorter fill and drain on large images).  With ramp > 0
// the first and the last `ramp` bands are shorter, halving towards both ends,
// so the first kernel starts after a short copy-in and the last copy-out is
// short too.  Bands go round-robin over the streams, so a band's copy-in waits
// at most behind the band nstreams places earlier.
std::vector<int> band_cuts(int rows, int ncbx, int band_cbs, int max_bands, int ramp) {
    long long nb = (long long)rows * ncbx / band_cbs;
    nb = nb < 1 ? 1 : (nb > max_bands ? max_bands : nb);
    if (nb > rows) nb = rows;
    const int len = (int)((rows + nb - 1) / nb);  // steady band length in rows
    std::vector<int> edge;                         // ramp lengths, shortest first
    for (int i = ramp; i >= 1; --i)
        if ((len >> i) >= 1) edge.push_back(len >> i);
    int e = 0;
    for (int l : edge) e += l;
    std::vector<int> lens;
    if (2 * e >= rows) {
        edge.clear();
        e = 0;
    }
    lens.insert(lens.end(), edge.begin(), edge.end());
    const int mid = rows - 2 * e;
    const int nmid = mid > 0 ? (mid + len - 1) / len : 0;
    for (int k = 0; k < nmid; k++) lens.push_back((int)((long long)mid * (k + 1) / nmid - (long long)mid * k / nmid));
    lens.insert(lens.end(), edge.rbegin(), edge.rend());
    std::vector<int> cuts{0};
    for (int l : lens)
        if (l > 0) cuts.push_back(cuts.back() + l);
    return cuts;
}

// Host-buffer coding through the reusable device buffers of the drop-in state.
int code_host_locked(DropInState &s, int direction, int *hdata, int X, int Y, const int *d_lut, int lut_n,
                     int passes, int levels, int cb) {
    if (!hdata || (direction != BPC_CODE && direction != BPC_DECODE)) return BPC_ERR_ARG;
    if (!valid_mode(passes, levels, cb) || !valid_geometry(X, Y, cb, levels) || !d_lut || lut_n <= 0)
        return BPC_ERR_ARG;
    const size_t n = (size_t)X * (size_t)Y;
    if (n > s.cap) {
        cudaFree(s.d_a);
        cudaFree(s.d_b);
        s.d_a = s.d_b = nullptr;
        s.cap = 0;
        CUDA_TRY(cudaMalloc((void **)&s.d_a, n * sizeof(int)));
        CUDA_TRY(cudaMalloc((void **)&s.d_b, n * sizeof(int)));
        s.cap = n;
    }
    if (!s.d_status) CUDA_TRY(cudaMalloc((void **)&s.d_status, sizeof(int)));
    const int nst = s.nstreams;
    for (int k = 0; k < nst; k++)
        if (!s.streams[k]) {
            CUDA_TRY(cudaStreamCreateWithFlags(&s.streams[k], cudaStreamNonBlocking));
            CUDA_TRY(cudaEventCreateWithFlags(&s.done[k], cudaEventDisableTiming));
        }
    CUDA_TRY(cudaMemsetAsync(s.d_status, 0, sizeof(int), s.streams[0]));
    CUDA_TRY(cudaEventRecord(s.done[0], s.streams[0]));
    for (int k = 1; k < nst; k++) CUDA_TRY(cudaStreamWaitEvent(s.streams[k], s.done[0], 0));
    const int ncbx = X / cb, rows = Y / cb;
    const std::vector<int> cuts = band_cuts(rows, ncbx, s.band_cbs, s.max_bands, s.ramp);
    const size_t row_words = (size_t)X * (size_t)cb;  // one codeblock row, either layout
    for (int k = 0; k + 1 < (int)cuts.size(); k++) {
        const int r0 = cuts[k], r1 = cuts[k + 1];
        cudaStream_t st = s.streams[k % nst];
        const size_t off = (size_t)r0 * row_words, cnt = (size_t)(r1 - r0) * row_words;
        CUDA_TRY(cudaMemcpyAsync(s.d_a + off, hdata + off, cnt * sizeof(int), cudaMemcpyHostToDevice, st));
        const int rc = bpc::code_device(direction == BPC_CODE, s.d_a, s.d_b, X, Y, d_lut, lut_n, passes, levels, cb,
                                   s.d_status, nullptr, 0, st, r0 * ncbx, r1 * ncbx);
        if (rc) return rc;
        CUDA_TRY(cudaMemcpyAsync(hdata + off, s.d_b + off, cnt * sizeof(int), cudaMemcpyDeviceToHost, st));
    }
    for (int k = 1; k < nst; k++) {
        CUDA_TRY(cudaEventRecord(s.done[k], s.streams[k]));
        CUDA_TRY(cudaStreamWaitEvent(s.streams[0], s.done[k], 0));
    }
    int st = 0;
    CUDA_TRY(cudaMemcpyAsync(&st, s.d_status, sizeof(int), cudaMemcpyDeviceToHost, s.streams[0]));
    CUDA_TRY(cudaStreamSynchronize(s.streams[0]));
    return st;
}

}  // namespace

namespace bpc {

int code_device(bool enc, const int *in, int *out, int X, int Y, const int *d_lut, int lut_n, int passes, int levels,
                int cb, int *d_status, int *d_counts, int grid, void *stream, int cb_begin, int cb_end, int *sched,
                bool latency_forms) {
    Params p;
    const int rc = fill_params(p, enc, in, out, X, Y, d_lut, lut_n, passes, levels, cb, d_status, d_counts);
    if (rc) return rc;
    if (cb_end >= 0) {
        p.cb_begin = cb_begin;
        p.cb_end = cb_end;
    }
    if (sched && grid <= 0) {
        const cudaError_t e = plan_order(enc, cb, p, sched, (cudaStream_t)stream, latency_forms);
        if (e != cudaSuccess) {
            std::fprintf(stderr, "bpc: work-order launch failed: %s\n", cudaGetErrorString(e));
            return BPC_ERR_CUDA;
        }
    }
    const cudaError_t e = launch_code(enc, passes, cb, p, grid, (cudaStream_t)stream, latency_forms);
    if (e != cudaSuccess) {
        std::fprintf(stderr, "bpc: kernel launch failed: %s\n", cudaGetErrorString(e));
        return BPC_ERR_CUDA;
    }
    return BPC_OK;
}

}  // namespace bpc

extern "C" {

int bpc_version(void) { return 100; }

const char *bpc_status_string(int st) {
    switch (st) {
        case BPC_OK: return "ok";
        case BPC_ERR_ARG: return "invalid argument";
        case BPC_ERR_CUDA: return "CUDA error";
        case BPC_ERR_FILE: return "cannot open LUT file";
        case BPC_ERR_PARSE: return "malformed LUT file";
        case BPC_ERR_NOMEM: return "out of memory";
        case BPC_ERR_TOO_LARGE: return "input larger than the fixed scratch or memory budget it must fit";
        case BPC_ERR_CANCELLED: return "request cancelled";
        default: break;
    }
    if (st > 0) {
        if (st & BPC_ST_SLOT_OVERFLOW) return "codeblock slot overflow";
        if (st & BPC_ST_BAD_STREAM) return "bad stream (MSB word outside 0..32)";
        if (st & BPC_ST_INPUT_RANGE) return "coefficient magnitude >= 2^28";
        if (st & BPC_ST_LUT_RANGE) return "LUT entry outside 0..255";
    }
    return "unknown status";
}

int bpc_set_mode(int passes, int dwt_levels, int cb_size) {
    if (!valid_mode(passes, dwt_levels, cb_size)) return BPC_ERR_ARG;
    DropInState &s = state();
    std::lock_guard<std::mutex> g(s.mu);
    s.passes = passes;
    s.levels = dwt_levels;
    s.cb = cb_size;
    return BPC_OK;
}

int bpc_get_mode(int *passes, int *dwt_levels, int *cb_size) {
    DropInState &s = state();
    std::lock_guard<std::mutex> g(s.mu);
    if (passes) *passes = s.passes;
    if (dwt_levels) *dwt_levels = s.levels;
    if (cb_size) *cb_size = s.cb;
    return BPC_OK;
}

int bpc_set_host_pipeline(int band_cbs, int max_bands, int streams, int ramp) {
    if (band_cbs < 1 || max_bands < 1 || max_bands > 4096 || streams < 1 || streams > DropInState::kMaxStreams ||
        ramp < 0 || ramp > 8)
        return BPC_ERR_ARG;
    DropInState &s = state();
    std::lock_guard<std::mutex> g(s.mu);
    s.band_cbs = band_cbs;
    s.max_bands = max_bands;
    s.nstreams = streams;
    s.ramp = ramp;
    return BPC_OK;
}

int bpc_get_host_pipeline(int *band_cbs, int *max_bands, int *streams, int *ramp) {
    DropInState &s = state();
    std::lock_guard<std::mutex> g(s.mu);
    if (band_cbs) *band_cbs = s.band_cbs;
    if (max_bands) *max_bands = s.max_bands;
    if (streams) *streams = s.nstreams;
    if (ramp) *ramp = s.ramp;
    return BPC_OK;
}

int bpc_host_band_rows(int X, int Y, int cb_size, int *starts, int capacity) {
    if ((cb_size != 64 && cb_size != 32) || !valid_geometry(X, Y, cb_size, 1) || capacity < 0) return BPC_ERR_ARG;
    DropInState &s = state();
    std::vector<int> cuts;
    {
        std::lock_guard<std::mutex> g(s.mu);
        cuts = band_cuts(Y / cb_size, X / cb_size, s.band_cbs, s.max_bands, s.ramp);
    }
    const int nb = (int)cuts.size() - 1;
    for (int k = 0; starts && k < nb && k < capacity; k++) starts[k] = cuts[k];
    return nb;
}

int bpc_last_status(void) {
    DropInState &s = state();
    std::lock_guard<std::mutex> g(s.mu);
    return s.last;
}

int bpc_lut_entries(int passes, int levels, int max_bitplane) {
    if ((passes != 2 && passes != 3) || levels < 1 || max_bitplane < 1) return BPC_ERR_ARG;
    return (int)bpc::lut_entries(passes, levels, max_bitplane);
}

int bpc_load_luts_host(const char *folder, int passes, int levels, int *out, int capacity, int *n_entries) {
    std::vector<int> lut;
    const int rc = bpc::load_luts_host(folder, passes, levels, lut);
    if (rc) return rc;
    if (n_entries) *n_entries = (int)lut.size();
    if (!out) return BPC_OK;
    if ((size_t)capacity < lut.size()) return BPC_ERR_ARG;
    for (size_t k = 0; k < lut.size(); k++) out[k] = lut[k];
    return BPC_OK;
}

int bpc_load_luts(const char *folder, int passes, int levels, int **d_lut, int *n_entries) {
    if (!d_lut) return BPC_ERR_ARG;
    *d_lut = nullptr;
    std::vector<int> lut;
    const int rc = bpc::load_luts_host(folder, passes, levels, lut);
    if (rc) return rc;
    int *d = nullptr;
    CUDA_TRY(cudaMalloc((void **)&d, lut.size() * sizeof(int)));
    const cudaError_t e = cudaMemcpy(d, lut.data(), lut.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(d);
        std::fprintf(stderr, "bpc: LUT upload failed: %s\n", cudaGetErrorString(e));
        return BPC_ERR_CUDA;
    }
    *d_lut = d;
    if (n_entries) *n_entries = (int)lut.size();
    DropInState &s = state();
    std::lock_guard<std::mutex> g(s.mu);
    s.lut_len[d] = (int)lut.size();
    return BPC_OK;
}

int bpc_lut_free(int *d_lut) {
    if (!d_lut) return BPC_OK;
    {
        DropInState &s = state();
        std::lock_guard<std::mutex> g(s.mu);
        s.lut_len.erase(d_lut);
    }
    CUDA_TRY(cudaFree(d_lut));
    return BPC_OK;
}

int bpc_code_host(int direction, int *hdata, int X, int Y, const int *d_lut, int lut_n, int passes, int levels,
                  int cb_size) {
    DropInState &s = state();
    std::lock_guard<std::mutex> g(s.mu);
    return code_host_locked(s, direction, hdata, X, Y, d_lut, lut_n, passes, levels, cb_size);
}

int bpc_encode_device(const int *d_coeffs, int *d_stream, int X, int Y, const int *d_lut, int lut_n, int passes,
                      int levels, int cb_size, int *d_status, int *d_counts, int grid, void *stream) {
    return bpc::code_device(true, d_coeffs, d_stream, X, Y, d_lut, lut_n, passes, levels, cb_size, d_status, d_counts, grid,
                       stream);
}

int bpc_decode_device(const int *d_stream, int *d_coeffs, int X, int Y, const int *d_lut, int lut_n, int passes,
                      int levels, int cb_size, int *d_status, int *d_counts, int grid, void *stream) {
    return bpc::code_device(false, d_stream, d_coeffs, X, Y, d_lut, lut_n, passes, levels, cb_size, d_status, d_counts,
                       grid, stream);
}

long long bpc_sched_ints(int X, int Y, int cb_size) {
    if ((cb_size != 64 && cb_size != 32) || !valid_geometry(X, Y, cb_size, 1)) return BPC_ERR_ARG;
    return bpc::sched_ints((X / cb_size) * (Y / cb_size), cb_size);
}

int bpc_encode_device_sched(const int *d_coeffs, int *d_stream, int X, int Y, const int *d_lut, int lut_n, int passes,
                            int levels, int cb_size, int *d_status, int *d_counts, int *d_sched, void *stream) {
    if (!d_sched) return BPC_ERR_ARG;
    return bpc::code_device(true, d_coeffs, d_stream, X, Y, d_lut, lut_n, passes, levels, cb_size, d_status, d_counts, 0,
                       stream, 0, -1, d_sched);
}

int bpc_decode_device_sched(const int *d_stream, int *d_coeffs, int X, int Y, const int *d_lut, int lut_n, int passes,
                            int levels, int cb_size, int *d_status, int *d_counts, int *d_sched, void *stream) {
    if (!d_sched) return BPC_ERR_ARG;
    return bpc::code_device(false, d_stream, d_coeffs, X, Y, d_lut, lut_n, passes, levels, cb_size, d_status, d_counts, 0,
                       stream, 0, -1, d_sched);
}

void load_LUTs(int **LUT, const char *folder) {
    int passes, levels;
    bpc_get_mode(&passes, &levels, nullptr);
    const int rc = bpc_load_luts(folder, passes, levels, LUT, nullptr);
    DropInState &s = state();
    std::lock_guard<std::mutex> g(s.mu);
    s.last = rc;
    if (rc) std::fprintf(stderr, "bpc: load_LUTs(%s): %s\n", folder ? folder : "(null)", bpc_status_string(rc));
}

void CUDA_BPC(int Direction, int *HData, int HDSize_X, int HDSize_Y, int *LUT) {
    DropInState &s = state();
    std::lock_guard<std::mutex> g(s.mu);
    int lut_n;
    auto it = s.lut_len.find(LUT);
    if (it != s.lut_len.end())
        lut_n = it->second;
    else  // a LUT this library did not load: assume the standard 15-bitplane layout
        lut_n = (int)bpc::lut_entries(s.passes, s.levels, 15);
    int rc = code_host_locked(s, Direction, HData, HDSize_X, HDSize_Y, LUT, lut_n, s.passes, s.levels, s.cb);
    // the reference releases the LUT after every call (BPC_PaCo.cu:1300)
    if (LUT) {
        s.lut_len.erase(LUT);
        const cudaError_t e = cudaFree(LUT);
        if (e != cudaSuccess && rc == BPC_OK) rc = BPC_ERR_CUDA;
    }
    s.last = rc;
    if (rc) std::fprintf(stderr, "bpc: CUDA_BPC: %s (%d)\n", bpc_status_string(rc), rc);
}

}  // extern "C"
