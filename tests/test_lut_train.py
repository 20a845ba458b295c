"""LUT training: symbol counts per LUT entry, the LUT files written from them,
and the tables they load as.  The CPU tests use the oracle's counts; the GPU
test holds the device counts equal to them."""
import os

import numpy as np
import pytest

import bpc_synth
from conftest import lut_folder


def probabilities(stats):
    n = stats[0::2].astype(np.float64)
    ones = stats[1::2].astype(np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        p = np.rint(128.0 * (n - ones) / n)
    return n, np.clip(np.nan_to_num(p, nan=64.0), 1, 127).astype(np.int32)


@pytest.mark.parametrize("passes", [2, 3])
def test_trained_tables_load_and_code(bpc, oracle_mod, passes, tmp_path):
    img = bpc_synth.synthetic_coefficients(512, 5, 31, amp=30, nrect=12)
    st = oracle_mod.lut_stats(img, passes, 5, 64)
    assert st.size == 2 * bpc.lib().bpc_lut_entries(passes, 5, 15)
    assert (st[1::2] <= st[0::2]).all()
    folder = str(tmp_path / "trained") + "/"
    bpc.lut_write(folder, st, passes, 5)
    names = ["ref.txt", "sig.txt", "sign.txt"] + (["cp_sig.txt", "cp_sign.txt"] if passes == 3 else [])
    assert sorted(os.listdir(folder)) == sorted(names)
    lut = bpc.load_luts_host(folder, passes, 5)
    np.testing.assert_array_equal(lut, oracle_mod.load_luts(folder, passes, 5))
    # every used entry below a group's last listed plane holds the trained value
    n, p = probabilities(st)
    used = np.nonzero(n)[0]
    assert used.size > 50
    agree = lut[used] == p[used]
    assert agree.mean() > 0.9, agree.mean()
    # the trained tables code the image they were trained on losslessly and
    # in fewer codewords than the shipped tables
    shipped = oracle_mod.load_luts(lut_folder(passes), passes, 5)
    s_t = oracle_mod.encode(img, lut, passes, 5, 64)
    s_s = oracle_mod.encode(img, shipped, passes, 5, 64)
    np.testing.assert_array_equal(oracle_mod.decode(s_t, img.shape, lut, passes, 5, 64), img)
    words = lambda s: int((s.reshape(-1, 4096)[:, 1:] != -1).sum())
    assert words(s_t) < words(s_s)


def test_group_layout(bpc, tmp_path):
    """Groups in layout order, planes up to one past the last used plane,
    that plane all 64; a group without data lists plane 0 only."""
    passes, levels = 2, 2
    n = bpc.lib().bpc_lut_entries(passes, levels, 15)
    st = np.zeros(2 * n, np.uint64)
    # ref section: group 1 (level 0 LH) plane 3 used, 10 symbols, 3 ones
    st[2 * (1 * 15 + 3)] = 10
    st[2 * (1 * 15 + 3) + 1] = 3
    folder = str(tmp_path) + "/"
    bpc.lut_write(folder, st, passes, levels)
    rows = [l.split() for l in open(folder + "ref.txt")]
    groups = [(int(r[0]), int(r[1])) for r in rows]
    assert groups[0] == (0, 0) and groups[-1] == (levels, 0)
    g1 = [r for r in rows if (int(r[0]), int(r[1])) == (0, 1)]
    assert [int(r[2]) for r in g1] == [0, 1, 2, 3, 4]
    assert int(g1[3][4]) == round(128 * 7 / 10) and int(g1[4][4]) == 64
    assert len([r for r in rows if (int(r[0]), int(r[1])) == (0, 0)]) == 1
    assert [int(r[2]) for r in rows if (int(r[0]), int(r[1])) == (levels, 0)] == list(range(15))


@pytest.mark.gpu
@pytest.mark.parametrize("passes,cb,levels", [(2, 64, 5), (3, 64, 5), (3, 32, 3), (2, 32, 6)])
def test_device_counts_equal_oracle(bpc, oracle_mod, passes, cb, levels):
    import torch
    a = bpc_synth.synthetic_coefficients(512, levels, 40 + levels, amp=30, nrect=12)
    b = bpc_synth.laplacian_coefficients(512, levels, 41)
    st = bpc.lut_stats(torch.from_numpy(a).cuda(), passes, levels, cb)
    bpc.lut_stats(torch.from_numpy(b).cuda(), passes, levels, cb, stats=st)
    torch.cuda.synchronize()
    want = oracle_mod.lut_stats(a, passes, levels, cb) + oracle_mod.lut_stats(b, passes, levels, cb)
    np.testing.assert_array_equal(st.cpu().numpy(), want)
