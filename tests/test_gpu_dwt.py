"""GPU 5/3 DWT against the numpy lifting (bpc_synth.dwt53): identical
coefficients, and the inverse restores the image."""
import numpy as np
import pytest

import bpc_synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("H,W,levels", [(256, 256, 5), (384, 256, 4), (512, 1024, 6), (64, 64, 1), (16, 16, 4),
                                         (24, 40, 2), (8, 2048, 3)])
def test_dwt_matches_numpy(bpc, H, W, levels):
    import torch
    rng = np.random.default_rng(H * W + levels)
    img = rng.integers(0, 256, size=(H, W)).astype(np.uint8)
    want = bpc_synth.dwt53(img, levels)
    d = torch.from_numpy(img.astype(np.int32) - 128).cuda()
    bpc.dwt53(d, levels)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d.cpu().numpy(), want)
    bpc.dwt53(d, levels, inverse=True)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d.cpu().numpy() + 128, img)


def test_gpu_generator_codes_losslessly(bpc, oracle_mod):
    import torch
    from conftest import lut_folder
    c = bpc_synth.synthetic_coefficients_gpu(512, 5, 3, amp=40)
    img = c.cpu().numpy()
    lut = oracle_mod.load_luts(lut_folder(3), 3, 5)
    s = oracle_mod.encode(img, lut, 3)
    np.testing.assert_array_equal(oracle_mod.decode(s, img.shape, lut, 3), img)
    assert np.abs(img).max() > 8
