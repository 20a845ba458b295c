"""Run the reference kernel (built by `make -C oracle ref` into oracle/_ref/)
on the GPU.  TEST INFRASTRUCTURE ONLY: the secondary oracle and the timing
bar for "the reference kernel rebuilt for the B200"; never part of the
product path.

Guards, so that the reference's kernel only touches memory it owns:
  * the LUT buffer is the loader array followed by zeros up to the largest
    index the reference forms (bitplane 32 of the LL group), so reads past
    the loader's array (BPC_PaCo.cu:233-249 with MSB >= 15) stay inside it;
  * every image is first encoded by the CPU oracle and refused if any
    codeblock has more codewords than its slot holds (the reference would
    write into the next slot or past the buffer, BPC_PaCo.cu:292);
  * only the `_sync`-shim builds (r2) run: in them the shuffles whose results
    are discarded on the first and last rows (BPC_PaCo.cu:644-704, inputs
    TData[-2..-1] and TData[128..129]) are removable builtins.
Dimensions must be multiples of 64 (the reference's own precondition).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
_libs = {}


def available(passes: int, variant: str = "r2") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libref_{variant}_p{passes}.so"))


def lib(passes: int, variant: str = "r2"):
    if not variant.startswith("r2"):
        raise ValueError("only the _sync-shim builds (r2*) are run")
    key = (passes, variant)
    if key not in _libs:
        L = ctypes.CDLL(os.path.join(REF_DIR, f"libref_{variant}_p{passes}.so"))
        L.ref_launch.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_void_p, ctypes.c_void_p]
        L.ref_launch.restype = ctypes.c_int
        L.ref_mode.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        p, l = ctypes.c_int(), ctypes.c_int()
        L.ref_mode(ctypes.byref(p), ctypes.byref(l))
        assert p.value == passes and l.value == 5, (p.value, l.value)
        _libs[key] = L
    return _libs[key]


def padded_lut(lut_np: np.ndarray, levels: int = 5) -> np.ndarray:
    nsig = 3 * 15 * 9 * levels + 135
    nsign = 3 * 15 * 4 * levels + 60
    a_sig = 3 * 15 * levels + 15
    a_sign = a_sig + nsig
    cp = nsig + nsign
    gmax = levels * 45 + 32
    need = max(a_sign + cp + gmax * 4 + 3, a_sig + cp + gmax * 9 + 8) + 1
    out = np.zeros(max(need, lut_np.size) + 64, np.int32)
    out[:lut_np.size] = lut_np
    return out


def check_no_overflow(img: np.ndarray, lut_np: np.ndarray, passes: int) -> np.ndarray:
    import oracle
    s, st = oracle.encode(img, lut_np, passes, 5, 64, with_status=True)
    if st.any():
        raise ValueError("refusing to run the reference kernel: a codeblock overflows its slot")
    return s


class RefCoder:
    """Device buffers for repeated reference launches of one image size."""

    def __init__(self, X: int, Y: int, lut_np: np.ndarray, passes: int, variant: str = "r2"):
        import torch
        assert X % 64 == 0 and Y % 64 == 0
        self.X, self.Y, self.passes = X, Y, passes
        self.L = lib(passes, variant)
        self.lut = torch.from_numpy(padded_lut(lut_np)).cuda()
        self.a = torch.empty(X * Y, dtype=torch.int32, device="cuda")
        self.b = torch.empty(X * Y, dtype=torch.int32, device="cuda")

    def launch(self, direction: int) -> None:
        rc = self.L.ref_launch(direction, self.a.data_ptr(), self.b.data_ptr(), self.X, self.Y,
                               self.lut.data_ptr(), None)
        if rc:
            raise RuntimeError(f"reference launch failed: cuda error {rc}")

    def run(self, direction: int, data: np.ndarray) -> np.ndarray:
        import torch
        self.a.copy_(torch.from_numpy(np.ascontiguousarray(data, np.int32).reshape(-1)))
        self.b.fill_(-1)  # cudaMemset(out, -1), BPC_PaCo.cu:1284
        torch.cuda.synchronize()
        self.launch(direction)
        torch.cuda.synchronize()
        return self.b.cpu().numpy()


def ref_encode(img: np.ndarray, lut_np: np.ndarray, passes: int, variant: str = "r2") -> np.ndarray:
    check_no_overflow(img, lut_np, passes)
    Y, X = img.shape
    return RefCoder(X, Y, lut_np, passes, variant).run(0, img)


def check_decodable(stream: np.ndarray, shape, lut_np: np.ndarray, passes: int) -> None:
    """The reference decoder reads one codeword per reservation; on a 3-pass
    all-zero codeblock (MSB word 32) it desynchronises (BPC_PaCo.cu:563-585)
    and may read past its slot, so such streams are refused, as are streams
    whose reservations overrun a slot in the oracle's reference-exact mode."""
    import oracle
    msb = np.asarray(stream).reshape(-1, 4096)[:, 0]
    if passes == 3 and (msb == 32).any():
        raise ValueError("refusing to run the reference decoder on a 3-pass all-zero codeblock")
    _, st = oracle.decode(stream, shape, lut_np, passes, 5, 64, ref_quirk=True, with_status=True)
    if st.any():
        raise ValueError("refusing to run the reference decoder: reservations overrun a slot")


def ref_decode(stream: np.ndarray, shape, lut_np: np.ndarray, passes: int, variant: str = "r2") -> np.ndarray:
    check_decodable(stream, shape, lut_np, passes)
    Y, X = shape
    return RefCoder(X, Y, lut_np, passes, variant).run(1, stream).reshape(Y, X)
