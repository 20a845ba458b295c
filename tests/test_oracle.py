"""The oracle (CPU restatement, oracle/bpc_oracle.c) pinned on the reference's
own known answers: the 1024 codeblock headers of the sample image and the
lossless round trip of main_example.cu:498-532, plus the LUT loader layout."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, REF_ROOT, lut_folder


def test_sample_headers_subset(oracle_mod, sample_subset):
    """(level, subband, MSBP) headers of the sample files == Find_Subband /
    Find_MSB (BPC_PaCo.cu:84-161) for the committed codeblocks."""
    tab = np.load(os.path.join(GOLDEN, "sample_headers.npy"))
    idx = np.load(os.path.join(GOLDEN, "sample_subset.npz"))["index"]
    for k in idx:
        _, lv, sb, msbp, x0, y0 = (int(v) for v in tab[k])
        assert oracle_mod.find_subband(x0, y0, 2048, 2048, 5) == (lv, sb)
        for passes in (2, 3):
            assert oracle_mod.block_msb(sample_subset, x0, y0, 64, passes) == msbp


@pytest.mark.skipif(not os.path.isdir(REF_ROOT), reason="reference checkout not present")
def test_sample_headers_full(oracle_mod):
    import make_fixtures
    img = make_fixtures.sample_image_full(REF_ROOT)
    tab = np.load(os.path.join(GOLDEN, "sample_headers.npy"))
    for _, lv, sb, msbp, x0, y0 in tab:
        assert oracle_mod.find_subband(int(x0), int(y0), 2048, 2048, 5) == (lv, sb)
        assert oracle_mod.block_msb(img, int(x0), int(y0), 64, 2) == msbp


@pytest.mark.parametrize("passes", [2, 3])
def test_lut_loader_layout(oracle_mod, passes):
    """load_LUTs layout (main_example.cu:219-448) for the shipped tables."""
    got = oracle_mod.load_luts(lut_folder(passes), passes, 5)
    want = np.load(os.path.join(GOLDEN, f"lut_naive_{passes}pass_L5.npy"))
    assert got.size == (3360 if passes == 2 else 6480)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("passes", [2, 3])
def test_sample_roundtrip_subset(oracle_mod, luts, sample_subset, passes):
    lut = luts(passes)
    s, st = oracle_mod.encode(sample_subset, lut, passes, with_status=True)
    assert st.max() == 0
    assert s.reshape(-1, 4096)[:, 0].min() >= 0
    d = oracle_mod.decode(s, sample_subset.shape, lut, passes)
    np.testing.assert_array_equal(d, sample_subset)


@pytest.mark.skipif(not os.path.isdir(REF_ROOT), reason="reference checkout not present")
@pytest.mark.parametrize("passes", [2, 3])
def test_sample_roundtrip_full(oracle_mod, luts, passes):
    """The reference's own test: encode, decode, compare (main_example.cu:518-532)."""
    import make_fixtures
    img = make_fixtures.sample_image_full(REF_ROOT)
    lut = luts(passes)
    s = oracle_mod.encode(img, lut, passes)
    np.testing.assert_array_equal(oracle_mod.decode(s, img.shape, lut, passes), img)


def test_all_zero_block_2pass(oracle_mod, luts):
    """MSB = 32 for an all-zero codeblock (32 - __ffs(__brev(0)), :159): 33
    planes are coded.  Codeblocks whose LUT reads run into zero entries emit
    a codeword per symbol and overflow; the others decode to zeros."""
    img = np.zeros((512, 512), np.int32)
    s, st = oracle_mod.encode(img, luts(2), 2, levels=5, with_status=True)
    assert (s.reshape(-1, 4096)[:, 0] == 32).all()
    assert (st == 0).sum() >= 60 and set(np.unique(st)) <= {0, oracle_mod.ST_OVERFLOW}
    d = oracle_mod.decode(s, img.shape, luts(2), 2, levels=5)
    for k in np.nonzero(st == 0)[0]:
        y0, x0 = (k // 8) * 64, (k % 8) * 64
        assert not d[y0:y0 + 64, x0:x0 + 64].any()


def test_all_zero_block_3pass_reference_decoder_desyncs(oracle_mod, luts):
    """3-pass all-zero codeblock: at b = 29 the CP pass codes the CP flag as a
    1 but the encoder does not make the coefficient significant (:523-530),
    while the reference decoder does and then reads a sign the encoder never
    wrote (:563-585).  The encoder-mirroring decoder reconstructs zeros."""
    img = np.zeros((512, 512), np.int32)
    lut = luts(3, 5)
    s, st = oracle_mod.encode(img, lut, 3, levels=5, with_status=True)
    ok = np.nonzero(st == 0)[0]
    assert len(ok) >= 60
    mirror = oracle_mod.decode(s, img.shape, lut, 3, levels=5)
    quirk = oracle_mod.decode(s, img.shape, lut, 3, levels=5, ref_quirk=True)
    differs = 0
    for k in ok:
        y0, x0 = (k // 8) * 64, (k % 8) * 64
        assert not mirror[y0:y0 + 64, x0:x0 + 64].any()
        differs += int(quirk[y0:y0 + 64, x0:x0 + 64].any())
    assert differs > 0


@pytest.mark.parametrize("passes", [2, 3])
def test_decoders_agree_on_regular_data(oracle_mod, luts, passes):
    import bpc_synth
    img = bpc_synth.synthetic_coefficients(256, 3, 5, amp=30)
    lut = luts(passes, 3)
    s = oracle_mod.encode(img, lut, passes, levels=3)
    a = oracle_mod.decode(s, img.shape, lut, passes, levels=3)
    b = oracle_mod.decode(s, img.shape, lut, passes, levels=3, ref_quirk=True)
    np.testing.assert_array_equal(a, img)
    np.testing.assert_array_equal(b, img)


@pytest.mark.parametrize("passes", [2, 3])
def test_cb32_roundtrip(oracle_mod, luts, passes):
    import bpc_synth
    img = bpc_synth.synthetic_coefficients(256, 4, 9, amp=40)
    lut = luts(passes, 4)
    s, st = oracle_mod.encode(img, lut, passes, levels=4, cb=32, with_status=True)
    assert st.max() == 0
    np.testing.assert_array_equal(oracle_mod.decode(s, img.shape, lut, passes, levels=4, cb=32), img)


def test_slot_overflow_flagged(oracle_mod):
    """More codewords than the slot holds (H5): flagged, never spills."""
    rng = np.random.default_rng(3)
    img = rng.integers(-(1 << 15), 1 << 15, size=(64, 128)).astype(np.int32)
    lut = np.full(3360, 127, np.int32)  # a 1 costs ~7 bits: many codewords
    s, st = oracle_mod.encode(img, lut, 2, levels=5, with_status=True)
    assert st[0] & oracle_mod.ST_OVERFLOW
    slots = s.reshape(-1, 4096)
    assert slots[1, 0] == oracle_mod.block_msb(img, 64, 0, 64, 2)  # next slot intact
