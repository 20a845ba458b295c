"""The C ABI library: loads, exports every function include/bpc_paco.h
declares, validates arguments, and its host LUT loader (no GPU calls)."""
import ctypes
import os
import re
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, lut_folder


def header_functions():
    text = open(os.path.join(ROOT, "include", "bpc_paco.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = "\n".join(l for l in text.splitlines() if not l.lstrip().startswith("#"))
    decl = r"^\s*(?:const\s+)?(?:void|int|char|long\s+long)\s*\**\s*([A-Za-z_]\w*)\s*\([^;{]*\)\s*;"
    return sorted(set(re.findall(decl, text, flags=re.M)))


def test_exports_every_declared_symbol(bpc):
    names = header_functions()
    assert {"CUDA_BPC", "load_LUTs", "bpc_encode_device", "bpc_decode_device"} <= set(names)
    L = bpc.lib()
    for n in names:
        assert hasattr(L, n), n
    assert set(bpc.EXPORTS) <= set(names)


def test_mode_validation(bpc):
    assert bpc.get_mode() == (2, 5, 64)
    assert bpc.lib().bpc_set_mode(4, 5, 64) == bpc.ERR_ARG
    assert bpc.lib().bpc_set_mode(2, 5, 48) == bpc.ERR_ARG
    bpc.set_mode(3, 6, 32)
    assert bpc.get_mode() == (3, 6, 32)
    bpc.set_mode(2, 5, 64)


def test_host_pipeline_validation(bpc):
    before = bpc.get_host_pipeline()
    assert before[0] >= 1 and before[1] >= 1 and 1 <= before[2] <= 16 and 0 <= before[3] <= 8
    for bad in ((0, 32, 8, 0), (512, 0, 8, 0), (512, 32, 0, 0), (512, 32, 17, 0), (512, 32, 8, -1), (512, 32, 8, 9)):
        assert bpc.lib().bpc_set_host_pipeline(*bad) == bpc.ERR_ARG
    assert bpc.get_host_pipeline() == before
    bpc.set_host_pipeline(128, 64, 16, 2)
    assert bpc.get_host_pipeline() == (128, 64, 16, 2)
    bpc.set_host_pipeline(*before)


@pytest.mark.parametrize("side,cb", [(64, 64), (2048, 64), (4096, 64), (4096, 32), (16384, 64), (3072, 64), (192, 32)])
@pytest.mark.parametrize("setting", [(512, 32, 8, 0), (256, 32, 16, 2), (128, 128, 16, 3), (64, 4096, 4, 8),
                                     (1, 1, 1, 0), (1 << 20, 32, 8, 2)])
def test_host_band_plan(bpc, side, cb, setting):
    """Bands tile the codeblock rows in order; the steady length follows the
    setting and the ramp bands halve towards both ends."""
    before = bpc.get_host_pipeline()
    try:
        bpc.set_host_pipeline(*setting)
        band_cbs, max_bands, _, ramp = setting
        rows, ncbx = side // cb, side // cb
        starts = bpc.host_band_rows(side, side, cb)
        lens = [b - a for a, b in zip(starts, starts[1:] + [rows])]
        assert starts[0] == 0 and all(l >= 1 for l in lens) and sum(lens) == rows
        nb = min(max(rows * ncbx // band_cbs, 1), max_bands, rows)
        steady = -(-rows // nb)
        assert max(lens) <= steady
        edge = [steady >> i for i in range(ramp, 0, -1) if steady >> i >= 1]
        if edge and 2 * sum(edge) < rows:
            assert lens[:len(edge)] == edge and lens[len(lens) - len(edge):] == edge[::-1]
        else:
            assert len(lens) == -(-rows // steady)
    finally:
        bpc.set_host_pipeline(*before)


def test_sched_ints(bpc):
    L = bpc.lib()
    # order and cost key per warp unit, then 4 ints for the isolated decode's queue counter
    assert L.bpc_sched_ints(4096, 4096, 64) == 2 * 4096 + 4
    assert L.bpc_sched_ints(4096, 4096, 32) == 2 * 8192 + 4
    assert L.bpc_sched_ints(96, 64, 32) == 2 * 3 + 4  # 6 codeblocks, 3 warp units
    for bad in ((100, 64, 64), (64, 64, 48), (0, 64, 64)):
        assert L.bpc_sched_ints(*bad) == bpc.ERR_ARG


def test_status_strings(bpc):
    assert bpc.status_string(0) == "ok"
    assert "overflow" in bpc.status_string(bpc.ST_SLOT_OVERFLOW)
    assert "LUT" in bpc.status_string(bpc.ERR_PARSE)


@pytest.mark.parametrize("passes", [2, 3])
def test_host_lut_loader_matches_layout(bpc, passes):
    got = bpc.load_luts_host(lut_folder(passes), passes, 5)
    want = np.load(os.path.join(GOLDEN, f"lut_naive_{passes}pass_L5.npy"))
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("levels", [1, 2, 3, 4, 6, 7])
@pytest.mark.parametrize("passes", [2, 3])
def test_host_lut_loader_other_levels_matches_oracle(bpc, oracle_mod, passes, levels):
    """DWT_LEVELS != 5 with the shipped 16-group files: truncated at the
    allocation (fewer levels) or zero-filled (more levels)."""
    np.testing.assert_array_equal(bpc.load_luts_host(lut_folder(passes), passes, levels),
                                  oracle_mod.load_luts(lut_folder(passes), passes, levels))


def test_lut_fill_rule(bpc, oracle_mod):
    """A group that lists planes 0..2 only: the fill writes 64 from entry
    2*N + 1 onward (overwriting contexts 1..N-1 of plane 2), the last group
    is not filled (main_example.cu:315-319)."""
    with tempfile.TemporaryDirectory() as d:
        rows = {"ref.txt": 1, "sig.txt": 9, "sign.txt": 4}
        for name, n in rows.items():
            with open(os.path.join(d, name), "w") as f:
                for g in range(2):
                    for bp in range(3):
                        vals = " ".join(str(10 + g * 20 + bp * 3 + k) for k in range(n))
                        f.write(f"0 {g} {bp} : {vals}\n")
        got = bpc.load_luts_host(d + "/", 2, 1)
        want = oracle_mod.load_luts(d + "/", 2, 1)
        np.testing.assert_array_equal(got, want)
        mb = 3
        sig0 = 3 * mb * 1 * 1 + mb  # ref section size for levels = 1
        assert got[sig0 + 2 * 9] == 10 + 6  # plane 2, context 0 kept
        assert (got[sig0 + 2 * 9 + 1: sig0 + 3 * 9] == 64).all()  # contexts 1..8 overwritten
        assert got[mb] == 30  # group 1, plane 0 of ref


def test_lut_loader_errors(bpc):
    n = ctypes.c_int()
    assert bpc.lib().bpc_load_luts_host(b"/nonexistent/", 2, 5, None, 0, ctypes.byref(n)) == bpc.ERR_FILE
    with tempfile.TemporaryDirectory() as d:
        for name in ("ref.txt", "sig.txt", "sign.txt"):
            open(os.path.join(d, name), "w").write("0 0 0 : 1 2\n0 0 x\n")
        assert bpc.lib().bpc_load_luts_host((d + "/").encode(), 2, 5, None, 0, ctypes.byref(n)) == bpc.ERR_PARSE


def test_device_entry_points_reject_bad_geometry(bpc):
    """Argument checks happen before any CUDA call."""
    vp = ctypes.c_void_p
    L = bpc.lib()
    for X, Y, cb in ((100, 64, 64), (64, 64, 48), (0, 64, 64)):
        rc = L.bpc_encode_device(vp(16), vp(16), X, Y, vp(16), 3360, 2, 5, cb, None, None, 0, None)
        assert rc == bpc.ERR_ARG
    assert L.bpc_decode_device(vp(16), vp(16), 64, 64, None, 3360, 2, 5, 64, None, None, 0, None) == bpc.ERR_ARG
    assert L.bpc_encode_device(vp(16), vp(16), 64, 64, vp(16), 3360, 4, 5, 64, None, None, 0, None) == bpc.ERR_ARG


def test_device_entry_points_reject_misaligned_inputs(bpc):
    """Coefficient inputs need 8-byte and slot-stream inputs 16-byte alignment
    (the kernels' vector loads); other pointers are refused before any CUDA
    call, valid geometry or not."""
    vp = ctypes.c_void_p
    L = bpc.lib()
    args = (64, 64, vp(4096), 3360, 2, 5, 64, None, None, 0, None)
    assert L.bpc_encode_device(vp(4096 + 4), vp(4096), *args) == bpc.ERR_ARG
    assert L.bpc_decode_device(vp(4096 + 8), vp(4096), *args) == bpc.ERR_ARG
    sargs = (64, 64, vp(4096), 3360, 2, 5, 64, None, None, vp(4096), None)
    assert L.bpc_encode_device_sched(vp(4096 + 4), vp(4096), *sargs) == bpc.ERR_ARG
    assert L.bpc_decode_device_sched(vp(4096 + 8), vp(4096), *sargs) == bpc.ERR_ARG
    assert L.bpc_encode_compact_noalloc(vp(4096 + 4), 64, 64, vp(4096), 3360, 2, 5, 64, vp(4096), vp(4096), None,
                                        None) == bpc.ERR_ARG
    assert L.bpc_lut_stats(vp(4096 + 4), 64, 64, 2, 5, 64, vp(4096), None) == bpc.ERR_ARG
