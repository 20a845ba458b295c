"""Parity of the sm_100a coder with the oracle: every stream word and every
decoded coefficient bit-exact, called through the C ABI."""
import numpy as np
import pytest

import bpc_synth
from conftest import lut_folder

pytestmark = pytest.mark.gpu


def synth(side, levels, seed, amp=20.0, nrect=30):
    return bpc_synth.synthetic_coefficients(side, levels, seed, amp=amp, nrect=nrect)


def check_roundtrip(bpc, oracle_mod, img, passes, levels, cb, lut_np=None):
    """Encode + decode on the GPU through bpc_code_host; compare with the oracle."""
    lut = bpc.DeviceLut(lut_folder(passes), passes, levels)
    try:
        if lut_np is None:
            lut_np = oracle_mod.load_luts(lut_folder(passes), passes, levels)
        want, wst = oracle_mod.encode(img, lut_np, passes, levels, cb, with_status=True)
        got, st = bpc.encode_host(img, lut, cb)
        bad = np.nonzero(got != want)[0]
        assert bad.size == 0, f"first stream mismatch at {bad[:8]} (slot {bad[0] // (cb * cb)})"
        assert st == int(np.bitwise_or.reduce(wst))
        dec, dst = bpc.decode_host(got, img.shape, lut, cb)
        wdec, wdst = oracle_mod.decode(want, img.shape, lut_np, passes, levels, cb, with_status=True)
        np.testing.assert_array_equal(dec, wdec)
        assert dst == int(np.bitwise_or.reduce(wdst))
        ok = np.nonzero(wst == 0)[0]
        ncbx = img.shape[1] // cb
        for k in ok[:: max(1, len(ok) // 64)]:
            y0, x0 = (k // ncbx) * cb, (k % ncbx) * cb
            np.testing.assert_array_equal(dec[y0:y0 + cb, x0:x0 + cb], img[y0:y0 + cb, x0:x0 + cb])
        return got, st
    finally:
        lut.close()


@pytest.mark.parametrize("passes", [2, 3])
def test_small_synthetic(bpc, oracle_mod, passes):
    img = synth(256, 5, 3, amp=40)
    _, st = check_roundtrip(bpc, oracle_mod, img, passes, 5, 64)
    assert st == 0


@pytest.mark.parametrize("passes", [2, 3])
def test_sample_subset(bpc, oracle_mod, sample_subset, passes):
    """The reference's sample codeblocks (MSB up to 12) at their positions;
    the other codeblocks are all-zero (MSB = 32)."""
    check_roundtrip(bpc, oracle_mod, sample_subset, passes, 5, 64)


def test_config1_2048_2pass(bpc, oracle_mod):
    img = synth(2048, 5, 1, amp=20, nrect=30)
    check_roundtrip(bpc, oracle_mod, img, 2, 5, 64)


def test_config2_4096_3pass(bpc, oracle_mod):
    img = synth(4096, 5, 2, amp=40, nrect=60)
    check_roundtrip(bpc, oracle_mod, img, 3, 5, 64)


@pytest.mark.parametrize("passes", [2, 3])
@pytest.mark.parametrize("levels", [3, 6])
def test_cb32(bpc, oracle_mod, passes, levels):
    img = synth(512, levels, 10 + levels, amp=30)
    check_roundtrip(bpc, oracle_mod, img, passes, levels, 32)


@pytest.mark.parametrize("passes", [2, 3])
def test_straddling_codeblocks(bpc, oracle_mod, passes):
    """3072 >> 5 = 96 is not a multiple of 64: codeblocks straddle subbands
    and lanes of one warp use different LUT groups."""
    img = synth(3072, 5, 21, amp=30)[:1024, :]
    check_roundtrip(bpc, oracle_mod, np.ascontiguousarray(img), passes, 5, 64)


@pytest.mark.parametrize("passes", [2, 3])
def test_all_zero_and_sparse(bpc, oracle_mod, passes):
    img = np.zeros((512, 512), np.int32)
    img[70, 3] = -1
    img[300, 301] = 5
    img[511, 511] = 1 << 20
    check_roundtrip(bpc, oracle_mod, img, passes, 5, 64)


@pytest.mark.parametrize("passes", [2, 3])
def test_laplacian_plane15(bpc, oracle_mod, passes):
    """Every magnitude plane up to 15 populated: LL codeblocks read LUT
    entries past the loader's array (zero padding)."""
    img = bpc_synth.laplacian_coefficients(512, 5, 4)
    img[0, 0] = 40000
    check_roundtrip(bpc, oracle_mod, img, passes, 5, 64)


def test_slot_overflow(bpc, oracle_mod):
    rng = np.random.default_rng(3)
    img = rng.integers(-(1 << 15), 1 << 15, size=(128, 128)).astype(np.int32)
    _, st = check_roundtrip(bpc, oracle_mod, img, 2, 5, 64)
    assert st & bpc.ST_SLOT_OVERFLOW


def test_device_api_and_persistent_grid(bpc, oracle_mod):
    import torch
    img = synth(1024, 5, 8, amp=40)
    lut_np = oracle_mod.load_luts(lut_folder(3), 3, 5)
    want = oracle_mod.encode(img, lut_np, 3, 5, 64)
    lut = bpc.DeviceLut(lut_folder(3), 3, 5)
    try:
        d_img = torch.from_numpy(img).cuda()
        outs = []
        for grid in (0, 37, 148):
            s = torch.full((img.size,), 12345, dtype=torch.int32, device="cuda")
            st = torch.zeros(1, dtype=torch.int32, device="cuda")
            cnt = torch.zeros(256, dtype=torch.int32, device="cuda")
            bpc.encode_device(d_img, s, lut, 64, st, cnt, grid)
            torch.cuda.synchronize()
            got = s.cpu().numpy()
            np.testing.assert_array_equal(got, want)
            assert st.item() == 0
            used = (want.reshape(-1, 4096)[:, 1:] != -1).sum(1)
            np.testing.assert_array_equal(cnt.cpu().numpy(), used)
            dec = torch.empty_like(d_img)
            bpc.decode_device(s, dec, lut, 64, st, None, grid)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(dec.cpu().numpy(), img)
            outs.append(got)
    finally:
        lut.close()


@pytest.mark.parametrize("cb", [64, 32])
def test_host_pipeline_settings(bpc, cb):
    """The host-buffer path gives the device path's stream and a lossless
    decode for every band plan: one band on one stream, many one-row bands,
    ramped bands, more bands than streams."""
    import torch
    img = synth(2048, 5, 21, amp=30, nrect=20)
    lut = bpc.DeviceLut(lut_folder(3), 3, 5)
    before = bpc.get_host_pipeline()
    try:
        d = torch.from_numpy(img).cuda()
        want = torch.empty_like(d)
        st = torch.zeros(1, dtype=torch.int32, device="cuda")
        bpc.encode_device(d, want, lut, cb, st)
        want = want.cpu().numpy().reshape(-1)
        for setting in ((1, 1, 1, 0), (1, 4096, 16, 0), (512, 32, 16, 3), (128, 7, 3, 1), (64, 4096, 2, 8)):
            bpc.set_host_pipeline(*setting)
            got, est = bpc.encode_host(img, lut, cb)
            assert est == 0
            np.testing.assert_array_equal(got, want, err_msg=str(setting))
            dec, dst = bpc.decode_host(got, img.shape, lut, cb)
            assert dst == 0
            np.testing.assert_array_equal(dec, img, err_msg=str(setting))
    finally:
        bpc.set_host_pipeline(*before)
        lut.close()


@pytest.mark.parametrize("side,levels,passes,cb", [(8192, 5, 3, 64), (6144, 6, 2, 64), (6144, 5, 3, 32),
                                                     (2048, 5, 3, 64), (4096, 5, 3, 64), (3072, 5, 2, 64),
                                                     (5120, 4, 3, 64)])
def test_work_ordered_calls(bpc, side, levels, passes, cb):
    """The work-ordered entry points write the same stream and coefficients as
    the raster-order ones: images of many warp waves (sorted, 64x64 and 32x32
    with codeblocks straddling subbands), one within half a wave (unsorted) and
    decodes of one to two waves (4096, 3072, 5120: sorted and isolated, the 24
    heaviest codeblocks on SMs of their own, the rest from a queue).  Outputs
    start from a sentinel, so a codeblock the order skipped shows."""
    import torch
    lut = bpc.DeviceLut(lut_folder(passes), passes, levels)
    try:
        d = bpc_synth.synthetic_coefficients_gpu(side, levels, 31, amp=60.0, nrect=100)
        st = torch.zeros(4, dtype=torch.int32, device="cuda")  # plain enc, ordered enc, plain dec, ordered dec
        want = torch.empty_like(d)
        bpc.encode_device(d, want, lut, cb, st[0:1])
        sched = bpc.sched_buffer(side, side, cb)
        got = torch.full_like(d, 0x7F7F7F7F)
        bpc.encode_device(d, got, lut, cb, st[1:2], sched=sched)
        assert torch.equal(got, want)
        want_dec = torch.empty_like(d)
        bpc.decode_device(want, want_dec, lut, cb, st[2:3])
        dec = torch.full_like(d, 0x7F7F7F7F)
        bpc.decode_device(got, dec, lut, cb, st[3:4], sched=sched)
        assert torch.equal(dec, want_dec)
        s = st.cpu().tolist()
        assert s[0] == s[1] and s[2] == s[3] and s[0] & ~bpc.ST_SLOT_OVERFLOW == 0
        if s[0] == 0:
            assert torch.equal(dec, d)
    finally:
        lut.close()


def test_isolated_decode_damaged_streams(bpc, oracle_mod):
    """A 4096x4096 3-pass stream with damaged slots, LL codeblocks among them
    (garbage codewords, MSB words 28-32, slots without the -1 fill), decodes
    the same through the isolated work-ordered call, the plain call and the
    oracle: coefficients and status bits.  The damage also changes the cost
    order the isolated call plans from."""
    import torch
    side, levels, passes, cb = 4096, 5, 3, 64
    lut = bpc.DeviceLut(lut_folder(passes), passes, levels)
    try:
        lut_np = oracle_mod.load_luts(lut_folder(passes), passes, levels)
        d = bpc_synth.synthetic_coefficients_gpu(side, levels, 43, amp=60.0, nrect=100)
        s_dev = torch.empty_like(d)
        st = torch.zeros(3, dtype=torch.int32, device="cuda")
        bpc.encode_device(d, s_dev, lut, cb, st[0:1])
        slots = s_dev.cpu().numpy().reshape(-1, cb * cb).copy()
        rng = np.random.default_rng(11)
        ncb = slots.shape[0]
        for k in (0, 1, 64, 65):  # LL codeblocks: garbage in their first used words
            used = int(np.argmax(slots[k] == -1)) or cb * cb
            slots[k, 1:used // 2] = rng.integers(0, 1 << 16, used // 2 - 1)
        pick = rng.choice(np.arange(66, ncb), 48, replace=False)
        for i, k in enumerate(pick):
            if i % 4 == 0:
                slots[k, 0] = 28 + (i // 4) % 4  # MSB words no encoder writes (28..31)
            elif i % 4 == 1:
                slots[k, 0] = 32  # all-zero claim over real codewords
            elif i % 4 == 2:
                slots[k, 1:] = rng.integers(0, 1 << 16, cb * cb - 1)  # no -1 fill
            else:
                slots[k, 1:9] = rng.integers(0, 1 << 16, 8)
        damaged = slots.reshape(-1)
        want, wst = oracle_mod.decode(damaged, (side, side), lut_np, passes, levels, cb, with_status=True)
        s_in = torch.from_numpy(damaged).cuda()
        plain = torch.full_like(d, 0x7F7F7F7F)
        bpc.decode_device(s_in, plain, lut, cb, st[1:2])
        iso = torch.full_like(d, 0x7F7F7F7F)
        bpc.decode_device(s_in, iso, lut, cb, st[2:3], sched=bpc.sched_buffer(side, side, cb))
        np.testing.assert_array_equal(plain.cpu().numpy(), want)
        np.testing.assert_array_equal(iso.cpu().numpy(), want)
        w = int(np.bitwise_or.reduce(wst))
        assert w & bpc.ST_BAD_STREAM
        assert st[1].item() == w and st[2].item() == w
    finally:
        lut.close()


def test_drop_in_flow(bpc, oracle_mod, sample_subset):
    """main_example.cu:498-532: load_LUTs, CUDA_BPC(CODE), load_LUTs again
    (CUDA_BPC frees it), CUDA_BPC(DECODE), compare."""
    for passes in (2, 3):
        bpc.set_mode(passes, 5, 64)
        h = sample_subset.copy().reshape(-1)
        lut = bpc.load_LUTs(lut_folder(passes))
        assert lut
        assert bpc.CUDA_BPC(bpc.CODE, h, 2048, 2048, lut) == 0
        want = oracle_mod.encode(sample_subset, oracle_mod.load_luts(lut_folder(passes), passes, 5), passes)
        np.testing.assert_array_equal(h, want)
        lut = bpc.load_LUTs(lut_folder(passes))
        assert bpc.CUDA_BPC(bpc.DECODE, h, 2048, 2048, lut) == 0
        np.testing.assert_array_equal(h.reshape(2048, 2048), sample_subset)
    bpc.set_mode(2, 5, 64)
