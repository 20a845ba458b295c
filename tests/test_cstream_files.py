"""Per-codeblock stream files (.bin, 16-bit big-endian, load_Data numbering):
written and read back on the host, byte layout checked against the reference's
reader (main_example.cu:51-68) and file order (:71-179).  No GPU."""
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN, lut_folder

sys.path.insert(0, GOLDEN)
import make_fixtures  # noqa: E402  (codeblock placement of load_Data)


@pytest.fixture(scope="module")
def sample_stream(oracle_mod, sample_subset):
    lut = oracle_mod.load_luts(lut_folder(3), 3, 5)
    return oracle_mod.encode(sample_subset, lut, 3, 5, 64)


def test_file_count(bpc):
    L = bpc.lib()
    assert L.bpc_cstream_files(2048, 2048, 5, 64) == 1024
    assert L.bpc_cstream_files(4096, 4096, 5, 64) == 4096
    assert L.bpc_cstream_files(512, 512, 3, 32) == 256
    assert L.bpc_cstream_files(100, 512, 3, 32) == bpc.ERR_ARG


def test_write_layout_and_read_back(bpc, sample_stream, tmp_path):
    folder = str(tmp_path) + "/"
    bpc.save_cstreams(folder, sample_stream, 2048, 2048, 5, 64)
    files = os.listdir(tmp_path)
    assert len(files) == 1024
    pos = make_fixtures.sample_placement(2048, 2048, 5, 64)
    slots = sample_stream.reshape(-1, 4096)
    for k in (0, 1, 63, 64, 500, 1023):
        x0, y0 = pos[k]
        want = slots[(y0 // 64) * 32 + x0 // 64].astype(np.int64) & 0xFFFF
        raw = np.fromfile(os.path.join(folder, f"{k}.bin"), dtype=">u2")
        np.testing.assert_array_equal(raw, want)
    back = bpc.load_cstreams(folder, 2048, 2048, 5, 64)
    want = np.where(sample_stream == -1, 65535, sample_stream)  # the fill reads back as 0xFFFF
    np.testing.assert_array_equal(back, want)


def test_reloaded_stream_decodes_the_same(bpc, oracle_mod, sample_stream, sample_subset, tmp_path):
    folder = str(tmp_path) + "/"
    bpc.save_cstreams(folder, sample_stream, 2048, 2048, 5, 64)
    back = bpc.load_cstreams(folder, 2048, 2048, 5, 64)
    lut = oracle_mod.load_luts(lut_folder(3), 3, 5)
    np.testing.assert_array_equal(oracle_mod.decode(back, (2048, 2048), lut, 3, 5, 64), sample_subset)


def test_short_and_missing_files(bpc, tmp_path):
    folder = str(tmp_path) + "/"
    s = np.arange(256 * 256, dtype=np.int32) & 0x7FFF
    bpc.save_cstreams(folder, s, 256, 256, 2, 64)
    with open(os.path.join(folder, "3.bin"), "r+b") as f:
        f.truncate(2 * 100 + 1)  # 100 whole words and half of the next
    back = bpc.load_cstreams(folder, 256, 256, 2, 64)
    pos = make_fixtures.sample_placement(256, 256, 2, 64)
    x0, y0 = pos[3]
    slot = back.reshape(-1, 4096)[(y0 // 64) * 4 + x0 // 64]
    want = s.reshape(-1, 4096)[(y0 // 64) * 4 + x0 // 64]
    np.testing.assert_array_equal(slot[:100], want[:100])
    assert (slot[100:] == -1).all()
    os.remove(os.path.join(folder, "7.bin"))
    with pytest.raises(bpc.BpcError):
        bpc.load_cstreams(folder, 256, 256, 2, 64)
