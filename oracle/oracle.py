"""ctypes binding of the CPU oracle (bpc_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py (cpu_baseline leg and the --impl reference arm) as the checker.  The
product library never imports this module.

The oracle restates the reference coder of PabloEnfedaque/CUDA_BPC-PaCo
(source/BPC_PaCo.cu:14-1224) and its LUT loader (source/main_example.cu:219-448).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

ST_OVERFLOW = 1
ST_BAD_STREAM = 2
ST_INPUT_RANGE = 4


def build() -> str:
    """Compile bpc_oracle.c into oracle/liboracle.so (gcc, no GPU needed)."""
    src = os.path.join(_HERE, "bpc_oracle.c")
    if (not os.path.exists(_LIB_PATH)) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-shared", "-fPIC", "-pthread", src, "-o", _LIB_PATH])
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        i32p = ctypes.POINTER(ctypes.c_int32)
        L.bpco_load_luts.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, i32p, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_int)]
        L.bpco_load_luts.restype = ctypes.c_int
        L.bpco_encode.argtypes = [i32p, i32p, ctypes.c_int, ctypes.c_int, i32p, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int, ctypes.c_int, i32p, ctypes.c_long, ctypes.c_long]
        L.bpco_encode.restype = ctypes.c_int
        L.bpco_decode.argtypes = [i32p, i32p, ctypes.c_int, ctypes.c_int, i32p, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int, ctypes.c_int, i32p, ctypes.c_int, ctypes.c_long,
                                  ctypes.c_long]
        L.bpco_decode.restype = ctypes.c_int
        lp = ctypes.POINTER(ctypes.c_long)
        for f in (L.bpco_encode_list, L.bpco_decode_list):
            f.argtypes = [i32p, i32p, ctypes.c_int, ctypes.c_int, i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                          ctypes.c_int, ctypes.c_int, i32p, lp, ctypes.c_long]
            f.restype = ctypes.c_int
        L.bpco_find_subband.argtypes = [ctypes.c_int] * 5 + [ctypes.POINTER(ctypes.c_int)] * 2
        L.bpco_find_subband.restype = None
        L.bpco_block_msb.argtypes = [i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.bpco_block_msb.restype = ctypes.c_int
        L.bpco_lut_stats.argtypes = [i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_void_p, ctypes.c_long]
        L.bpco_lut_stats.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def load_luts(folder: str, passes: int, levels: int = 5) -> np.ndarray:
    """load_LUTs (main_example.cu:219-448) over a zero-initialised buffer."""
    if not folder.endswith("/"):
        folder += "/"
    n = ctypes.c_int(0)
    rc = lib().bpco_load_luts(folder.encode(), passes, levels, None, 0, ctypes.byref(n))
    if rc:
        raise OSError(f"oracle LUT load failed ({rc}) for {folder}")
    out = np.zeros(n.value, np.int32)
    rc = lib().bpco_load_luts(folder.encode(), passes, levels, _p(out), n.value, ctypes.byref(n))
    if rc:
        raise OSError(f"oracle LUT load failed ({rc}) for {folder}")
    return out


def encode(img: np.ndarray, lut: np.ndarray, passes: int, levels: int = 5, cb: int = 64, threads: int = 0,
           cb_range=(0, -1), with_status: bool = False):
    img = np.ascontiguousarray(img, dtype=np.int32)
    Y, X = img.shape
    lut = np.ascontiguousarray(lut, dtype=np.int32)
    out = np.full(img.size, -1, np.int32)
    st = np.zeros((X // cb) * (Y // cb), np.int32)
    rc = lib().bpco_encode(_p(img), _p(out), X, Y, _p(lut), lut.size, passes, levels, cb,
                           threads or os.cpu_count() or 1, _p(st), cb_range[0], cb_range[1])
    if rc < 0:
        raise ValueError(f"oracle encode: bad arguments ({rc})")
    return (out, st) if with_status else out


def decode(stream: np.ndarray, shape, lut: np.ndarray, passes: int, levels: int = 5, cb: int = 64,
           threads: int = 0, ref_quirk: bool = False, cb_range=(0, -1), with_status: bool = False):
    Y, X = shape
    stream = np.ascontiguousarray(stream, dtype=np.int32).reshape(-1)
    assert stream.size == X * Y
    lut = np.ascontiguousarray(lut, dtype=np.int32)
    out = np.zeros((Y, X), np.int32)
    st = np.zeros((X // cb) * (Y // cb), np.int32)
    rc = lib().bpco_decode(_p(stream), _p(out), X, Y, _p(lut), lut.size, passes, levels, cb,
                           threads or os.cpu_count() or 1, _p(st), int(ref_quirk), cb_range[0], cb_range[1])
    if rc < 0:
        raise ValueError(f"oracle decode: bad arguments ({rc})")
    return (out, st) if with_status else out


def code_list(enc: bool, data: np.ndarray, shape, lut: np.ndarray, passes: int, levels: int, cb: int,
              cb_list, out: np.ndarray | None = None, threads: int = 0):
    """Encode (enc) or decode only the codeblocks in cb_list (raster indices)
    of an X x Y image or slot stream.  `out` (X*Y int32, reused if given)
    receives their slots / pixels; everything else in it is left untouched.
    Returns (out, status per codeblock)."""
    Y, X = shape
    data = np.ascontiguousarray(data, dtype=np.int32).reshape(-1)
    assert data.size == X * Y
    lut = np.ascontiguousarray(lut, dtype=np.int32)
    if out is None:
        out = np.full(X * Y, -1 if enc else 0, np.int32)
    assert out.dtype == np.int32 and out.size == X * Y and out.flags["C_CONTIGUOUS"]
    lst = np.ascontiguousarray(cb_list, dtype=np.int64)
    st = np.zeros((X // cb) * (Y // cb), np.int32)
    f = lib().bpco_encode_list if enc else lib().bpco_decode_list
    rc = f(_p(data), _p(out.reshape(-1)), X, Y, _p(lut), lut.size, passes, levels, cb, threads or os.cpu_count() or 1,
           _p(st), lst.ctypes.data_as(ctypes.POINTER(ctypes.c_long)), lst.size)
    if rc < 0:
        raise ValueError(f"oracle {'encode' if enc else 'decode'} list: bad arguments ({rc})")
    return out, st


def find_subband(x: int, y: int, X: int, Y: int, levels: int):
    a, b = ctypes.c_int(0), ctypes.c_int(0)
    lib().bpco_find_subband(x, y, X, Y, levels, ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


def block_msb(img: np.ndarray, x0: int, y0: int, cb: int, passes: int) -> int:
    img = np.ascontiguousarray(img, dtype=np.int32)
    return lib().bpco_block_msb(_p(img), img.shape[1], x0, y0, cb, passes)


def lut_entries(passes: int, levels: int, planes: int = 15) -> int:
    """Entries of the load_LUTs layout: sections ref, sig, sign [, cp_sig,
    cp_sign] of 3 * planes * N * levels + planes * N ints each."""
    ns = [1, 9, 4] + ([9, 4] if passes == 3 else [])
    return sum(3 * planes * n * levels + planes * n for n in ns)


def lut_stats(img: np.ndarray, passes: int, levels: int = 5, cb: int = 64, threads: int = 0) -> np.ndarray:
    """LUT training counts of one image: uint64 array of 2 * lut_entries,
    [2k] symbols coded with entry k, [2k+1] of them equal to 1 (planes 0..14)."""
    img = np.ascontiguousarray(img, dtype=np.int32)
    Y, X = img.shape
    n = lut_entries(passes, levels)
    st = np.zeros(2 * n, np.uint64)
    rc = lib().bpco_lut_stats(_p(img), X, Y, passes, levels, cb, threads or os.cpu_count() or 1, st.ctypes.data, n)
    if rc < 0:
        raise ValueError(f"oracle lut_stats: bad arguments ({rc})")
    return st
