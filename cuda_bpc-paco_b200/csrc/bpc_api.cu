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
    // host-buffer calls run bands of codeblock rows on these streams so that
    // the copies in both directions overlap the kernels
    static constexpr int kStreams = 8;
    cudaStream_t streams[kStreams] = {};
    cudaEvent_t done[kStreams] = {};
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

int fill_params(bpc::Params &p, const int *in, int *out, int X, int Y, const int *d_lut, int lut_n, int passes,
                int levels, int cb, int *d_status, int *d_counts) {
    if (!valid_mode(passes, levels, cb) || !valid_geometry(X, Y, cb, levels) || !in || !out || !d_lut || lut_n <= 0)
        return BPC_ERR_ARG;
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

int code_device(bool enc, const int *in, int *out, int X, int Y, const int *d_lut, int lut_n, int passes, int levels,
                int cb, int *d_status, int *d_counts, int grid, void *stream, int cb_begin = 0, int cb_end = -1) {
    bpc::Params p;
    const int rc = fill_params(p, in, out, X, Y, d_lut, lut_n, passes, levels, cb, d_status, d_counts);
    if (rc) return rc;
    if (cb_end >= 0) {
        p.cb_begin = cb_begin;
        p.cb_end = cb_end;
    }
    const cudaError_t e = bpc::launch_code(enc, passes, cb, p, grid, (cudaStream_t)stream);
    if (e != cudaSuccess) {
        std::fprintf(stderr, "bpc: kernel launch failed: %s\n", cudaGetErrorString(e));
        return BPC_ERR_CUDA;
    }
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
    if (!s.streams[0])
        for (int k = 0; k < DropInState::kStreams; k++) {
            CUDA_TRY(cudaStreamCreateWithFlags(&s.streams[k], cudaStreamNonBlocking));
            CUDA_TRY(cudaEventCreateWithFlags(&s.done[k], cudaEventDisableTiming));
        }
    CUDA_TRY(cudaMemsetAsync(s.d_status, 0, sizeof(int), s.streams[0]));
    CUDA_TRY(cudaEventRecord(s.done[0], s.streams[0]));
    for (int k = 1; k < DropInState::kStreams; k++) CUDA_TRY(cudaStreamWaitEvent(s.streams[k], s.done[0], 0));
    // bands of codeblock rows: the input rows and the output slots of a band
    // are contiguous in both layouts (coefficients row-major, slots in raster
    // order of codeblocks)
    const int ncbx = X / cb, rows = Y / cb;
    // bands of at least 512 codeblocks (each band's kernel still spreads over
    // the SMs), at most 32 (shorter pipeline fill and drain on large images);
    // bands go round-robin over the 8 streams, so a band's copy-in waits at
    // most behind the band 8 places earlier
    const long long ncb = (long long)ncbx * rows;
    int nband = (int)(ncb / 512);
    nband = nband < 1 ? 1 : (nband > 32 ? 32 : nband);
    if (nband > rows) nband = rows;
    const size_t row_words = (size_t)X * (size_t)cb;  // one codeblock row, either layout
    for (int k = 0; k < nband; k++) {
        const int r0 = (int)((long long)rows * k / nband), r1 = (int)((long long)rows * (k + 1) / nband);
        if (r1 <= r0) continue;
        cudaStream_t st = s.streams[k % DropInState::kStreams];
        const size_t off = (size_t)r0 * row_words, cnt = (size_t)(r1 - r0) * row_words;
        CUDA_TRY(cudaMemcpyAsync(s.d_a + off, hdata + off, cnt * sizeof(int), cudaMemcpyHostToDevice, st));
        const int rc = code_device(direction == BPC_CODE, s.d_a, s.d_b, X, Y, d_lut, lut_n, passes, levels, cb,
                                   s.d_status, nullptr, 0, st, r0 * ncbx, r1 * ncbx);
        if (rc) return rc;
        CUDA_TRY(cudaMemcpyAsync(hdata + off, s.d_b + off, cnt * sizeof(int), cudaMemcpyDeviceToHost, st));
    }
    for (int k = 1; k < DropInState::kStreams; k++) {
        CUDA_TRY(cudaEventRecord(s.done[k], s.streams[k]));
        CUDA_TRY(cudaStreamWaitEvent(s.streams[0], s.done[k], 0));
    }
    int st = 0;
    CUDA_TRY(cudaMemcpyAsync(&st, s.d_status, sizeof(int), cudaMemcpyDeviceToHost, s.streams[0]));
    CUDA_TRY(cudaStreamSynchronize(s.streams[0]));
    return st;
}

}  // namespace

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
    return code_device(true, d_coeffs, d_stream, X, Y, d_lut, lut_n, passes, levels, cb_size, d_status, d_counts, grid,
                       stream);
}

int bpc_decode_device(const int *d_stream, int *d_coeffs, int X, int Y, const int *d_lut, int lut_n, int passes,
                      int levels, int cb_size, int *d_status, int *d_counts, int grid, void *stream) {
    return code_device(false, d_stream, d_coeffs, X, Y, d_lut, lut_n, passes, levels, cb_size, d_status, d_counts,
                       grid, stream);
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
