"""The product's coder source (cuda_bpc-paco_b200/csrc/bpc_core.cuh) compiled for
the host and run with one user-level context per lane (tests/emu/emu_warp.cpp),
checked bit-exact against the oracle: streams, decodes, status bits and LUT
statistics.  No GPU; the same source the sm_100a kernels are built from."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import bpc_synth
from conftest import ROOT, lut_folder


@pytest.fixture(scope="module")
def emu(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("emu") / "libemu.so")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I",
                           os.path.join(ROOT, "cuda_bpc-paco_b200", "csrc"),
                           os.path.join(ROOT, "tests", "emu", "emu_warp.cpp"), "-o", out])
    L = ctypes.CDLL(out)
    vp = ctypes.c_void_p
    L.emu_code.argtypes = [ctypes.c_int] * 4 + [vp, vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int,
                                                  vp, vp]
    L.emu_code.restype = ctypes.c_int
    return L


def run(emu, enc, img_or_stream, shape, lut, passes, levels, cb, kind=0, stats=None, offsets=None):
    Y, X = shape
    src = np.ascontiguousarray(img_or_stream, dtype=np.int32).reshape(-1)
    out = np.zeros(X * Y, np.int32)
    rc = emu.emu_code(enc, kind, passes, cb, src.ctypes.data, out.ctypes.data, X, Y, lut.ctypes.data, lut.size,
                      levels, None if stats is None else stats.ctypes.data,
                      None if offsets is None else offsets.ctypes.data)
    assert rc >= 0, "lanes of a warp met different collectives"
    return out, rc


def roundtrip(emu, oracle_mod, img, passes, levels, cb):
    """Every form of the coder loops (kind 0; the latency forms, kinds 2 and 3:
    two and three encoder positions per iteration) against the oracle:
    streams, decodes, status bits."""
    lut = oracle_mod.load_luts(lut_folder(passes), passes, levels)
    want, wst = oracle_mod.encode(img, lut, passes, levels, cb, with_status=True)
    wdec, wdst = oracle_mod.decode(want, img.shape, lut, passes, levels, cb, with_status=True)
    for kind in (0, 2, 3):
        got, st = run(emu, 1, img, img.shape, lut, passes, levels, cb, kind=kind)
        np.testing.assert_array_equal(got, want)
        assert st == int(np.bitwise_or.reduce(wst))
        dec, dst = run(emu, 0, got, img.shape, lut, passes, levels, cb, kind=kind)
        np.testing.assert_array_equal(dec.reshape(img.shape), wdec)
        assert dst == int(np.bitwise_or.reduce(wdst))
    return st


@pytest.mark.parametrize("passes", [2, 3])
@pytest.mark.parametrize("cb", [64, 32])
def test_synthetic(emu, oracle_mod, passes, cb):
    img = bpc_synth.synthetic_coefficients(256, 5, 3, amp=40)
    assert roundtrip(emu, oracle_mod, img, passes, 5, cb) == 0


@pytest.mark.parametrize("passes", [2, 3])
def test_straddling_and_sparse(emu, oracle_mod, passes):
    img = np.ascontiguousarray(bpc_synth.synthetic_coefficients(3072, 5, 21, amp=30)[:64, :384])
    roundtrip(emu, oracle_mod, img, passes, 5, 64)
    z = np.zeros((128, 128), np.int32)
    z[70, 3] = -1
    z[127, 127] = 1 << 20
    roundtrip(emu, oracle_mod, z, passes, 5, 64)


def test_plane15_and_overflow(emu, oracle_mod):
    img = bpc_synth.laplacian_coefficients(128, 5, 4)
    img[0, 0] = 40000
    roundtrip(emu, oracle_mod, img, 3, 5, 64)
    rng = np.random.default_rng(3)
    noisy = rng.integers(-(1 << 15), 1 << 15, size=(64, 64)).astype(np.int32)
    assert roundtrip(emu, oracle_mod, noisy, 2, 5, 64) & 1  # slot overflow, dropped like the oracle


@pytest.mark.parametrize("passes,cb", [(3, 64), (2, 32)])
def test_lut_statistics(emu, oracle_mod, passes, cb):
    img = bpc_synth.synthetic_coefficients(128, 5, 12, amp=30)
    lut = oracle_mod.load_luts(lut_folder(passes), passes, 5)
    n = oracle_mod.lut_entries(passes, 5)
    st = np.zeros(2 * n, np.uint64)
    run(emu, 1, img, img.shape, lut, passes, 5, cb, kind=1, stats=st)
    np.testing.assert_array_equal(st, oracle_mod.lut_stats(img, passes, 5, cb))


@pytest.mark.parametrize("passes,cb", [(3, 64), (2, 32)])
def test_decode_from_compact_container(emu, oracle_mod, passes, cb):
    """The batched form's container (MSB + codewords per codeblock, int64
    offsets, words past a codeblock read as the -1 fill) decodes like the slot
    stream."""
    img = bpc_synth.synthetic_coefficients(128, 5, 13, amp=30)
    lut = oracle_mod.load_luts(lut_folder(passes), passes, 5)
    slots = oracle_mod.encode(img, lut, passes, 5, cb).reshape(-1, cb * cb)
    sizes = np.minimum((slots[:, 1:] != -1).sum(1) + 1, cb * cb)
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    compact = np.concatenate([slots[g, :sizes[g]] for g in range(len(sizes))]).astype(np.int32)
    buf = np.zeros(img.size, np.int32)
    buf[:compact.size] = compact
    dec, _ = run(emu, 0, buf, img.shape, lut, passes, 5, cb, offsets=offsets)
    np.testing.assert_array_equal(dec.reshape(img.shape), img)


def test_compact_container_damaged_offsets(emu, oracle_mod):
    """Offsets that point outside the container, or decrease, are damage: the
    codeblock decodes as a bad stream (zeros, status bit 2) without reading
    outside the container, and the other codeblocks decode intact."""
    img = bpc_synth.synthetic_coefficients(128, 5, 13, amp=30)
    lut = oracle_mod.load_luts(lut_folder(3), 3, 5)
    slots = oracle_mod.encode(img, lut, 3, 5, 64).reshape(-1, 64 * 64)
    sizes = np.minimum((slots[:, 1:] != -1).sum(1) + 1, 64 * 64)
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    compact = np.concatenate([slots[g, :sizes[g]] for g in range(len(sizes))]).astype(np.int32)
    buf = np.zeros(img.size, np.int32)
    buf[:compact.size] = compact
    bad = offsets.copy()
    bad[3] = img.size + 10**9       # codeblock 2 ends, codeblock 3 starts, past the container
    dec, st = run(emu, 0, buf, img.shape, lut, 3, 5, 64, offsets=bad)
    assert st & 2
    blocks = dec.reshape(2, 64, 2, 64).transpose(0, 2, 1, 3).reshape(4, 64, 64)
    want = img.reshape(2, 64, 2, 64).transpose(0, 2, 1, 3).reshape(4, 64, 64)
    np.testing.assert_array_equal(blocks[:2], want[:2])
    assert not blocks[2].any() and not blocks[3].any()
    bad = offsets.copy()
    bad[1] = -5                     # negative start
    dec, st = run(emu, 0, buf, img.shape, lut, 3, 5, 64, offsets=bad)
    assert st & 2
    blocks = dec.reshape(2, 64, 2, 64).transpose(0, 2, 1, 3).reshape(4, 64, 64)
    np.testing.assert_array_equal(blocks[2:], want[2:])
