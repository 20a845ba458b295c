"""Python binding of the codec's C ABI (include/bpc_paco.h).

It mirrors the reference's host interface (source/main_example.cu:8 CUDA_BPC,
:219 load_LUTs) and exposes the device-pointer entry points for callers that
keep data on the GPU (torch tensors are accepted there; torch is only used for
device memory and streams).  The library is the in-tree libbpc_paco.so; if it
is missing this module raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbpc_paco.so")

CODE, DECODE = 0, 1
OK = 0
ERR_ARG, ERR_CUDA, ERR_FILE, ERR_PARSE, ERR_NOMEM, ERR_TOO_LARGE, ERR_CANCELLED = -1, -2, -3, -4, -5, -6, -7
ST_SLOT_OVERFLOW, ST_BAD_STREAM, ST_INPUT_RANGE, ST_LUT_RANGE = 1, 2, 4, 8

EXPORTS = ("CUDA_BPC", "load_LUTs", "bpc_set_mode", "bpc_get_mode", "bpc_last_status", "bpc_status_string",
           "bpc_load_luts_host", "bpc_load_luts", "bpc_lut_free", "bpc_code_host", "bpc_encode_device",
           "bpc_decode_device", "bpc_lut_entries", "bpc_version")

_lib = None


class BpcError(RuntimeError):
    pass


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise BpcError(f"{LIB_PATH} is missing: build it with `python cuda_bpc-paco_b200/build.py`")
        L = ctypes.CDLL(LIB_PATH)
        ip = ctypes.POINTER(ctypes.c_int)
        vp = ctypes.c_void_p
        L.CUDA_BPC.argtypes = [ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, vp]
        L.CUDA_BPC.restype = None
        L.load_LUTs.argtypes = [ctypes.POINTER(vp), ctypes.c_char_p]
        L.load_LUTs.restype = None
        L.bpc_set_mode.argtypes = [ctypes.c_int] * 3
        L.bpc_get_mode.argtypes = [ip, ip, ip]
        L.bpc_last_status.argtypes = []
        L.bpc_status_string.argtypes = [ctypes.c_int]
        L.bpc_status_string.restype = ctypes.c_char_p
        L.bpc_load_luts_host.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, ip]
        L.bpc_load_luts.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp), ip]
        L.bpc_lut_free.argtypes = [vp]
        L.bpc_code_host.argtypes = [ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int]
        dev = [vp, vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp,
               ctypes.c_int, vp]
        L.bpc_encode_device.argtypes = dev
        L.bpc_decode_device.argtypes = dev
        L.bpc_sched_ints.argtypes = [ctypes.c_int] * 3
        L.bpc_sched_ints.restype = ctypes.c_longlong
        dev_s = [vp, vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp,
                 vp, vp]
        L.bpc_encode_device_sched.argtypes = dev_s
        L.bpc_decode_device_sched.argtypes = dev_s
        L.bpc_encode_device_sched.restype = ctypes.c_int
        L.bpc_decode_device_sched.restype = ctypes.c_int
        L.bpc_lut_entries.argtypes = [ctypes.c_int] * 3
        L.bpc_set_host_pipeline.argtypes = [ctypes.c_int] * 4
        L.bpc_get_host_pipeline.argtypes = [ip, ip, ip, ip]
        L.bpc_host_band_rows.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int]
        for f in ("bpc_set_host_pipeline", "bpc_get_host_pipeline", "bpc_host_band_rows", "bpc_set_mode", "bpc_get_mode", "bpc_last_status", "bpc_load_luts_host", "bpc_load_luts",
                  "bpc_lut_free", "bpc_code_host", "bpc_encode_device", "bpc_decode_device", "bpc_lut_entries",
                  "bpc_version"):
            getattr(L, f).restype = ctypes.c_int
        _lib = L
    return _lib


def status_string(st: int) -> str:
    return lib().bpc_status_string(st).decode()


def _check(rc: int, what: str) -> int:
    if rc < 0:
        raise BpcError(f"{what}: {status_string(rc)} ({rc})")
    return rc


def _folder(folder: str) -> bytes:
    return (folder if folder.endswith("/") else folder + "/").encode()


# ----------------------------------------------------------------- drop-in
def set_mode(passes: int, levels: int = 5, cb: int = 64) -> None:
    _check(lib().bpc_set_mode(passes, levels, cb), "bpc_set_mode")


def get_mode():
    a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    lib().bpc_get_mode(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
    return a.value, b.value, c.value


def set_host_pipeline(band_cbs: int, max_bands: int, streams: int, ramp: int = 0) -> None:
    """Bands of >= band_cbs codeblocks, <= max_bands of them, on `streams` CUDA
    streams for the host-buffer calls, the first and last `ramp` bands halving
    towards the ends (speed only; outputs do not change)."""
    _check(lib().bpc_set_host_pipeline(band_cbs, max_bands, streams, ramp), "bpc_set_host_pipeline")


def get_host_pipeline():
    v = [ctypes.c_int() for _ in range(4)]
    lib().bpc_get_host_pipeline(*[ctypes.byref(x) for x in v])
    return tuple(x.value for x in v)


def host_band_rows(X: int, Y: int, cb: int = 64) -> list:
    """First codeblock row of each band the host-buffer calls cut an X x Y image into."""
    n = _check(lib().bpc_host_band_rows(X, Y, cb, None, 0), "bpc_host_band_rows")
    buf = (ctypes.c_int * max(n, 1))()
    lib().bpc_host_band_rows(X, Y, cb, buf, n)
    return list(buf[:n])


def load_LUTs(folder: str) -> int:
    """Reference load_LUTs: returns the device pointer (int), 0 on error."""
    p = ctypes.c_void_p()
    lib().load_LUTs(ctypes.byref(p), _folder(folder))
    return p.value or 0


def CUDA_BPC(direction: int, hdata: np.ndarray, X: int, Y: int, lut_ptr: int) -> int:
    """Reference CUDA_BPC: codes `hdata` (int32, X*Y, C-contiguous) in place;
    frees the LUT.  Returns bpc_last_status()."""
    assert hdata.dtype == np.int32 and hdata.flags["C_CONTIGUOUS"] and hdata.size == X * Y
    lib().CUDA_BPC(direction, hdata.ctypes.data, X, Y, ctypes.c_void_p(lut_ptr))
    return lib().bpc_last_status()


# -------------------------------------------------------- explicit variants
def load_luts_host(folder: str, passes: int, levels: int = 5) -> np.ndarray:
    n = ctypes.c_int(0)
    _check(lib().bpc_load_luts_host(_folder(folder), passes, levels, None, 0, ctypes.byref(n)), "load_luts_host")
    out = np.zeros(n.value, np.int32)
    _check(lib().bpc_load_luts_host(_folder(folder), passes, levels, out.ctypes.data, out.size, ctypes.byref(n)),
           "load_luts_host")
    return out


class DeviceLut:
    """A LUT resident on the device (bpc_load_luts / bpc_lut_free)."""

    def __init__(self, folder: str, passes: int, levels: int = 5):
        p, n = ctypes.c_void_p(), ctypes.c_int(0)
        _check(lib().bpc_load_luts(_folder(folder), passes, levels, ctypes.byref(p), ctypes.byref(n)), "load_luts")
        self.ptr, self.n, self.passes, self.levels = p.value, n.value, passes, levels

    def close(self) -> None:
        if self.ptr:
            lib().bpc_lut_free(ctypes.c_void_p(self.ptr))
            self.ptr = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def encode_host(img: np.ndarray, lut: DeviceLut, cb: int = 64) -> tuple[np.ndarray, int]:
    buf = np.ascontiguousarray(img, dtype=np.int32).copy()
    Y, X = buf.shape
    st = _check(lib().bpc_code_host(CODE, buf.ctypes.data, X, Y, ctypes.c_void_p(lut.ptr), lut.n, lut.passes,
                                    lut.levels, cb), "bpc_code_host")
    return buf.reshape(-1), st


def decode_host(stream: np.ndarray, shape, lut: DeviceLut, cb: int = 64) -> tuple[np.ndarray, int]:
    Y, X = shape
    buf = np.ascontiguousarray(stream, dtype=np.int32).reshape(-1).copy()
    assert buf.size == X * Y
    st = _check(lib().bpc_code_host(DECODE, buf.ctypes.data, X, Y, ctypes.c_void_p(lut.ptr), lut.n, lut.passes,
                                    lut.levels, cb), "bpc_code_host")
    return buf.reshape(Y, X), st


def _ptr(t) -> int:
    return 0 if t is None else int(t.data_ptr())


def sched_buffer(X: int, Y: int, cb: int = 64):
    """Device scratch for the work-ordered calls (bpc_sched_ints ints)."""
    import torch
    n = _check(lib().bpc_sched_ints(X, Y, cb), "bpc_sched_ints")
    return torch.empty(max(n, 1), dtype=torch.int32, device="cuda")


def encode_device(coeffs, stream_out, lut: DeviceLut, cb: int = 64, status=None, counts=None, grid: int = 0,
                  cuda_stream: int | None = None, sched=None) -> None:
    """Device-to-device encode of torch int32 tensors (Y x X coeffs -> X*Y
    stream), enqueued on `cuda_stream` (default: torch's current stream).
    With `sched` (sched_buffer) large images are coded in work order."""
    import torch
    Y, X = coeffs.shape
    s = torch.cuda.current_stream().cuda_stream if cuda_stream is None else cuda_stream
    if sched is not None:
        _check(lib().bpc_encode_device_sched(_ptr(coeffs), _ptr(stream_out), X, Y, ctypes.c_void_p(lut.ptr), lut.n,
                                             lut.passes, lut.levels, cb, ctypes.c_void_p(_ptr(status)),
                                             ctypes.c_void_p(_ptr(counts)), ctypes.c_void_p(_ptr(sched)),
                                             ctypes.c_void_p(s)), "bpc_encode_device_sched")
        return
    _check(lib().bpc_encode_device(_ptr(coeffs), _ptr(stream_out), X, Y, ctypes.c_void_p(lut.ptr), lut.n, lut.passes,
                                   lut.levels, cb, ctypes.c_void_p(_ptr(status)), ctypes.c_void_p(_ptr(counts)), grid,
                                   ctypes.c_void_p(s)), "bpc_encode_device")


def decode_device(stream_in, coeffs_out, lut: DeviceLut, cb: int = 64, status=None, counts=None, grid: int = 0,
                  cuda_stream: int | None = None, sched=None) -> None:
    import torch
    Y, X = coeffs_out.shape
    s = torch.cuda.current_stream().cuda_stream if cuda_stream is None else cuda_stream
    if sched is not None:
        _check(lib().bpc_decode_device_sched(_ptr(stream_in), _ptr(coeffs_out), X, Y, ctypes.c_void_p(lut.ptr),
                                             lut.n, lut.passes, lut.levels, cb, ctypes.c_void_p(_ptr(status)),
                                             ctypes.c_void_p(_ptr(counts)), ctypes.c_void_p(_ptr(sched)),
                                             ctypes.c_void_p(s)), "bpc_decode_device_sched")
        return
    _check(lib().bpc_decode_device(_ptr(stream_in), _ptr(coeffs_out), X, Y, ctypes.c_void_p(lut.ptr), lut.n,
                                   lut.passes, lut.levels, cb, ctypes.c_void_p(_ptr(status)),
                                   ctypes.c_void_p(_ptr(counts)), grid, ctypes.c_void_p(s)), "bpc_decode_device")


# ------------------------------------------------------------ batched form
class Batch:
    """Batched persistent coding of many images (bpc_batch_* in the C ABI).

    images: list of (X, Y, levels, passes, cb); luts: dict passes -> folder.
    Device tensors are torch int32; the compact container is one int32 tensor
    plus int64 offsets (codeblocks + 1 entries)."""

    def __init__(self, images, luts: dict):
        import torch
        L = lib()
        vp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)
        L.bpc_batch_create.argtypes = [ctypes.c_int, ip, ip, ip, ip, ip, ctypes.POINTER(vp), ip, ctypes.POINTER(vp)]
        L.bpc_batch_codeblocks.argtypes = [vp]
        L.bpc_batch_codeblocks.restype = ctypes.c_longlong
        L.bpc_batch_words.argtypes = [vp]
        L.bpc_batch_words.restype = ctypes.c_longlong
        L.bpc_batch_encode.argtypes = [vp, ctypes.POINTER(vp), vp, vp, vp, vp]
        L.bpc_batch_decode.argtypes = [vp, vp, vp, ctypes.POINTER(vp), vp, vp]
        L.bpc_batch_set_schedule.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.bpc_batch_get_schedule.argtypes = [vp, ip, ip, ip, ip]
        L.bpc_batch_set_tuning.argtypes = [vp] + [ctypes.c_int] * 6
        L.bpc_batch_get_tuning.argtypes = [vp] + [ip] * 6
        L.bpc_batch_tune.argtypes = [vp, ctypes.POINTER(vp), vp, vp, ctypes.POINTER(vp), vp,
                                     ctypes.POINTER(ctypes.c_double)]
        L.bpc_batch_destroy.argtypes = [vp]
        self.images = list(images)
        n = len(self.images)
        arr = lambda k: (ctypes.c_int * n)(*[im[k] for im in self.images])
        self._luts = {}
        lut_ptrs, lut_ns = [], []
        for (_, _, lv, ps, _) in self.images:
            if (ps, lv) not in self._luts:
                self._luts[(ps, lv)] = DeviceLut(luts[ps], ps, lv)
            d = self._luts[(ps, lv)]
            lut_ptrs.append(d.ptr)
            lut_ns.append(d.n)
        h = vp()
        _check(L.bpc_batch_create(n, arr(0), arr(1), arr(2), arr(3), arr(4), (vp * n)(*lut_ptrs),
                                  (ctypes.c_int * n)(*lut_ns), ctypes.byref(h)), "bpc_batch_create")
        self.h = h
        self.codeblocks = L.bpc_batch_codeblocks(h)
        self.words = L.bpc_batch_words(h)
        self.torch = torch

    def _ptrs(self, tensors):
        return (ctypes.c_void_p * len(tensors))(*[t.data_ptr() for t in tensors])

    def encode(self, coeffs, compact, offsets, status=None, stream=None):
        s = self.torch.cuda.current_stream().cuda_stream if stream is None else stream
        _check(lib().bpc_batch_encode(self.h, self._ptrs(coeffs), compact.data_ptr(), offsets.data_ptr(),
                                      None if status is None else status.data_ptr(), s), "bpc_batch_encode")

    def decode(self, compact, offsets, out, status=None, stream=None):
        s = self.torch.cuda.current_stream().cuda_stream if stream is None else stream
        _check(lib().bpc_batch_decode(self.h, compact.data_ptr(), offsets.data_ptr(), self._ptrs(out),
                                      None if status is None else status.data_ptr(), s), "bpc_batch_decode")

    def set_schedule(self, ctas_enc: int, ctas_dec: int, per_item: int, graph: bool = True) -> None:
        _check(lib().bpc_batch_set_schedule(self.h, ctas_enc, ctas_dec, per_item, int(graph)), "set_schedule")

    def schedule(self):
        a, b, c, d = (ctypes.c_int() for _ in range(4))
        lib().bpc_batch_get_schedule(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(d))
        return a.value, b.value, c.value, bool(d.value)

    def set_tuning(self, warps_enc: int = 4, warps_dec: int = 4, cost_enc: bool = False, cost_dec: bool = False,
                   seq_enc: bool = False, seq_dec: bool = False):
        _check(lib().bpc_batch_set_tuning(self.h, warps_enc, warps_dec, int(cost_enc), int(cost_dec), int(seq_enc),
                                          int(seq_dec)), "set_tuning")

    def tuning(self):
        v = [ctypes.c_int() for _ in range(6)]
        lib().bpc_batch_get_tuning(self.h, *[ctypes.byref(x) for x in v])
        return v[0].value, v[1].value, bool(v[2].value), bool(v[3].value), bool(v[4].value), bool(v[5].value)

    def tune(self, coeffs, compact, offsets, out) -> float:
        us = ctypes.c_double()
        s = self.torch.cuda.current_stream().cuda_stream
        _check(lib().bpc_batch_tune(self.h, self._ptrs(coeffs), compact.data_ptr(), offsets.data_ptr(),
                                    self._ptrs(out), s, ctypes.byref(us)), "bpc_batch_tune")
        return us.value

    def close(self):
        if getattr(self, "h", None):
            lib().bpc_batch_destroy(self.h)
            self.h = None
        for d in self._luts.values():
            d.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def slots_to_compact(stream: np.ndarray, cb: int) -> list:
    """Per-codeblock [MSB, codewords...] word lists of a slot stream."""
    s = np.asarray(stream).reshape(-1, cb * cb)
    out = []
    for row in s:
        n = int(np.count_nonzero(row[1:] != -1))
        out.append(row[:1 + n])
    return out


def encode_compact_noalloc(coeffs, compact, offsets, lut: DeviceLut, cb: int = 64, status=None,
                           cuda_stream: int | None = None) -> int:
    """One-image encode into the compact container without allocating
    (bpc_encode_compact_noalloc): for callers that may not allocate device
    memory while they code.  Returns the C status (negative on error)."""
    import torch
    L = lib()
    vp = ctypes.c_void_p
    L.bpc_encode_compact_noalloc.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_int, vp, vp, vp, vp]
    L.bpc_encode_compact_noalloc.restype = ctypes.c_int
    Y, X = coeffs.shape
    s = torch.cuda.current_stream().cuda_stream if cuda_stream is None else cuda_stream
    return L.bpc_encode_compact_noalloc(_ptr(coeffs), X, Y, vp(lut.ptr), lut.n, lut.passes, lut.levels, cb,
                                        _ptr(compact), _ptr(offsets), vp(_ptr(status)), vp(s))


def dwt53(data, levels: int, inverse: bool = False, tmp=None, cuda_stream: int | None = None) -> None:
    """In-place reversible 5/3 DWT of a torch int32 (Y x X) tensor on the GPU
    (bpc_dwt53_forward / _inverse)."""
    import torch
    L = lib()
    vp = ctypes.c_void_p
    f = L.bpc_dwt53_inverse if inverse else L.bpc_dwt53_forward
    f.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp]
    f.restype = ctypes.c_int
    Y, X = data.shape
    t = torch.empty_like(data) if tmp is None else tmp
    s = torch.cuda.current_stream().cuda_stream if cuda_stream is None else cuda_stream
    _check(f(vp(data.data_ptr()), X, Y, levels, vp(t.data_ptr()), vp(s)), "bpc_dwt53")


def save_cstreams(folder: str, stream: np.ndarray, X: int, Y: int, levels: int = 5, cb: int = 64) -> None:
    """Write a host slot stream as per-codeblock .bin files (bpc_save_cstreams)."""
    s = np.ascontiguousarray(stream, dtype=np.int32)
    assert s.size == X * Y
    L = lib()
    L.bpc_save_cstreams.argtypes = [ctypes.c_char_p, ctypes.c_void_p] + [ctypes.c_int] * 4
    _check(L.bpc_save_cstreams(_folder(folder), s.ctypes.data, X, Y, levels, cb), "bpc_save_cstreams")


def load_cstreams(folder: str, X: int, Y: int, levels: int = 5, cb: int = 64, fill: int = -1) -> np.ndarray:
    """Read per-codeblock .bin files into a slot stream (bpc_load_cstreams);
    slots no file covers keep `fill`."""
    s = np.full(X * Y, fill, np.int32)
    L = lib()
    L.bpc_load_cstreams.argtypes = [ctypes.c_char_p, ctypes.c_void_p] + [ctypes.c_int] * 4
    _check(L.bpc_load_cstreams(_folder(folder), s.ctypes.data, X, Y, levels, cb), "bpc_load_cstreams")
    return s


def lut_stats(coeffs, passes: int, levels: int = 5, cb: int = 64, stats=None):
    """LUT training counts of device coefficients (bpc_lut_stats), added to
    `stats` (a torch uint64 tensor of 2 * bpc_lut_entries(passes, levels, 15),
    created zeroed when None); returns it."""
    import torch
    L = lib()
    vp = ctypes.c_void_p
    L.bpc_lut_stats.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp]
    n = L.bpc_lut_entries(passes, levels, 15)
    if stats is None:
        stats = torch.zeros(2 * n, dtype=torch.uint64, device=coeffs.device)
    assert stats.numel() == 2 * n
    Y, X = coeffs.shape
    s = torch.cuda.current_stream().cuda_stream
    _check(L.bpc_lut_stats(_ptr(coeffs), X, Y, passes, levels, cb, _ptr(stats), vp(s)), "bpc_lut_stats")
    return stats


def lut_write(folder: str, stats: np.ndarray, passes: int, levels: int = 5) -> None:
    """Write LUT text files from host training counts (bpc_lut_write)."""
    st = np.ascontiguousarray(stats, dtype=np.uint64)
    L = lib()
    L.bpc_lut_write.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    assert st.size == 2 * L.bpc_lut_entries(passes, levels, 15)
    os.makedirs(folder, exist_ok=True)
    _check(L.bpc_lut_write(_folder(folder), st.ctypes.data, passes, levels), "bpc_lut_write")


class Server:
    """The request server (bpc_server_*): encode and decode requests of mixed
    size admitted in arrival order against a device-memory budget reserved
    once, overlapped on up to `max_in_flight` streams by a native worker
    thread.  Inputs are device tensors the caller keeps alive until their
    request completes; outputs live in the server's budget until released."""

    def __init__(self, budget_bytes: int, max_in_flight: int = 8):
        L = lib()
        vp, ll = ctypes.c_void_p, ctypes.c_longlong
        L.bpc_server_create.argtypes = [ll, ctypes.c_int, ctypes.POINTER(vp)]
        L.bpc_server_register_lut.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              ctypes.POINTER(ctypes.c_int)]
        L.bpc_server_submit.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.bpc_server_submit.restype = ll
        L.bpc_server_cancel.argtypes = [vp, ll]
        L.bpc_server_poll.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, ctypes.POINTER(ctypes.c_int)]
        L.bpc_server_release.argtypes = [vp, vp]
        L.bpc_server_state.argtypes = [vp] + [ctypes.POINTER(ll)] * 4
        L.bpc_server_destroy.argtypes = [vp]
        self.L = L
        h = vp()
        _check(L.bpc_server_create(budget_bytes, max_in_flight, ctypes.byref(h)), "bpc_server_create")
        self.h = h
        self._cap = 0
        self._grow(256)

    def _grow(self, n: int) -> None:
        if n > self._cap:
            self._cap = n
            self._t = np.zeros(n, np.int64)
            self._o = np.zeros(n, np.uint64)
            self._l = np.zeros(n, np.float64)
            self._s = np.zeros(n, np.int32)

    def register_lut(self, lut: DeviceLut) -> int:
        i = ctypes.c_int()
        _check(self.L.bpc_server_register_lut(self.h, ctypes.c_void_p(lut.ptr), lut.n, lut.passes, lut.levels,
                                              ctypes.byref(i)), "bpc_server_register_lut")
        return i.value

    def submit(self, direction: int, data, lut_id: int, cb: int = 64, shape=None) -> int:
        """Queue a request on device data (a torch tensor or a raw pointer
        with `shape` = (Y, X)); returns the ticket or a negative error."""
        Y, X = shape if shape is not None else data.shape
        ptr = data if isinstance(data, int) else data.data_ptr()
        return self.L.bpc_server_submit(self.h, direction, ctypes.c_void_p(ptr), X, Y, lut_id, cb)

    def cancel(self, ticket: int) -> int:
        return self.L.bpc_server_cancel(self.h, ticket)

    def poll(self, max_n: int = 256, wait_us: int = 0):
        """Finished requests as a list of (ticket, output pointer, latency us,
        status)."""
        self._grow(max_n)
        n = ctypes.c_int()
        _check(self.L.bpc_server_poll(self.h, max_n, wait_us, self._t.ctypes.data, self._o.ctypes.data,
                                      self._l.ctypes.data, self._s.ctypes.data, ctypes.byref(n)), "bpc_server_poll")
        k = n.value
        return list(zip(self._t[:k].tolist(), self._o[:k].tolist(), self._l[:k].tolist(), self._s[:k].tolist()))

    def release(self, output_ptr: int) -> None:
        _check(self.L.bpc_server_release(self.h, ctypes.c_void_p(output_ptr)), "bpc_server_release")

    def state(self) -> dict:
        v = [ctypes.c_longlong() for _ in range(4)]
        _check(self.L.bpc_server_state(self.h, *[ctypes.byref(x) for x in v]), "bpc_server_state")
        return dict(zip(("queued", "in_flight", "bytes_used", "completed"), (x.value for x in v)))

    def close(self) -> None:
        if self.h:
            self.L.bpc_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def as_tensor(ptr: int, n: int, device_index: int | None = None):
    """A torch int32 view of `n` ints of device memory at `ptr` (no copy);
    valid while the memory is (e.g. until the server output is released)."""
    import torch

    class _View:
        __cuda_array_interface__ = {"shape": (n,), "typestr": "<i4", "data": (ptr, False), "version": 3}

    dev = torch.cuda.current_device() if device_index is None else device_index
    return torch.as_tensor(_View(), device=f"cuda:{dev}")
