"""HBM-scale parity: the 16384 x 16384, 5-level, 3-pass workload (65,536
codeblocks of 64 x 64, 268 M coefficients, slot offsets up to 2^28 words)
on the GPU, checked against the oracle on a fixed sample of codeblocks: the
whole last codeblock row, the whole last codeblock column, the four LL
codeblocks and 2,000 random ones.  Both inputs of that workload: the
synthetic image (noise amplitude 80, 400 rectangles) and the i.i.d.
Laplacian field with bitplane 15 populated in every codeblock.  The plain
call and the work-ordered call must write the same stream; the GPU decode
must return the input; the oracle must write the GPU's slots for the sample
and decode them back to the input (the encode -> decode -> compare loop of
the reference's own check, main_example.cu:518-532, at full size)."""
import numpy as np
import pytest

import bpc_synth
from conftest import lut_folder

pytestmark = pytest.mark.gpu

SIDE, LEVELS, PASSES, CB = 16384, 5, 3, 64


def sample_codeblocks(ncbx, seed=5, n_random=2000):
    ncb = ncbx * ncbx
    last_row = np.arange(ncb - ncbx, ncb)
    last_col = np.arange(ncbx - 1, ncb, ncbx)
    ll = np.array([0, 1, ncbx, ncbx + 1])
    rnd = np.random.default_rng(seed).choice(ncb, n_random, replace=False)
    return np.unique(np.concatenate([last_row, last_col, ll, rnd]))


@pytest.mark.parametrize("kind", ["image", "laplacian"])
def test_cfg5_sample_vs_oracle(bpc, oracle_mod, kind):
    import torch
    if kind == "image":
        d_img = bpc_synth.synthetic_coefficients_gpu(SIDE, LEVELS, 1, amp=80.0, nrect=400)
    else:
        d_img = bpc_synth.laplacian_coefficients_gpu(SIDE, LEVELS, 1, cb=CB)
    N = SIDE * SIDE
    lut = bpc.DeviceLut(lut_folder(PASSES), PASSES, LEVELS)
    try:
        st = torch.zeros(1, dtype=torch.int32, device="cuda")
        d_s = torch.empty(N, dtype=torch.int32, device="cuda")
        bpc.encode_device(d_img, d_s, lut, CB, st)
        d_s2 = torch.empty(N, dtype=torch.int32, device="cuda")
        bpc.encode_device(d_img, d_s2, lut, CB, st, sched=bpc.sched_buffer(SIDE, SIDE, CB))
        torch.cuda.synchronize()
        assert st.item() == 0
        assert torch.equal(d_s, d_s2), "work-ordered encode differs from the plain call"
        del d_s2
        d_o = torch.empty_like(d_img)
        bpc.decode_device(d_s, d_o, lut, CB, st)
        torch.cuda.synchronize()
        assert st.item() == 0
        assert torch.equal(d_o, d_img), "GPU decode did not return the input"
        d_o.fill_(0)
        bpc.decode_device(d_s, d_o, lut, CB, st, sched=bpc.sched_buffer(SIDE, SIDE, CB))
        torch.cuda.synchronize()
        assert torch.equal(d_o, d_img), "work-ordered GPU decode did not return the input"
        del d_o
        img = d_img.cpu().numpy()
        got = d_s.cpu().numpy()
    finally:
        lut.close()
    lut_np = oracle_mod.load_luts(lut_folder(PASSES), PASSES, LEVELS)
    lst = sample_codeblocks(SIDE // CB)
    want, wst = oracle_mod.code_list(True, img, img.shape, lut_np, PASSES, LEVELS, CB, lst)
    assert not wst[lst].any()
    g, w = got.reshape(-1, CB * CB), want.reshape(-1, CB * CB)
    bad = [int(k) for k in lst if not np.array_equal(g[k], w[k])]
    assert not bad, f"{len(bad)} sampled slots differ from the oracle, first {bad[:8]}"
    dec, dst = oracle_mod.code_list(False, got, img.shape, lut_np, PASSES, LEVELS, CB, lst)
    assert not dst[lst].any()
    ncbx = SIDE // CB
    for k in lst:
        y0, x0 = (k // ncbx) * CB, (k % ncbx) * CB
        np.testing.assert_array_equal(dec[y0 * SIDE:(y0 + CB) * SIDE].reshape(CB, SIDE)[:, x0:x0 + CB],
                                      img[y0:y0 + CB, x0:x0 + CB])
