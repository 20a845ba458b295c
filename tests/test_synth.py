"""Synthetic input generator: the 5/3 DWT is reversible and seeded inputs are
reproducible."""
import numpy as np

import bpc_synth


def test_dwt_roundtrip():
    img = bpc_synth.make_image(256, 11)
    for levels in (1, 3, 5):
        c = bpc_synth.dwt53(img, levels)
        np.testing.assert_array_equal(bpc_synth.idwt53(c, levels), img)


def test_seeded():
    a = bpc_synth.synthetic_coefficients(128, 3, 4)
    b = bpc_synth.synthetic_coefficients(128, 3, 4)
    np.testing.assert_array_equal(a, b)
    assert a.dtype == np.int32 and a.shape == (128, 128)


def test_laplacian_planes():
    c = bpc_synth.laplacian_coefficients(256, 5, 1)
    assert np.abs(c).max() < (1 << 16)


def test_laplacian_every_codeblock_codes_16_planes():
    """The HBM-scale Laplacian input (run here with torch on the CPU): every
    64x64 codeblock's largest magnitude lies in plane 15."""
    c = bpc_synth.laplacian_coefficients_gpu(512, 5, 3, device="cpu").numpy()
    assert c.dtype == np.int32 and c.shape == (512, 512)
    m = np.abs(c).reshape(8, 64, 8, 64).max(axis=(1, 3))
    assert (m >= (1 << 15)).all() and (m < (1 << 16)).all()
    d = bpc_synth.laplacian_coefficients_gpu(512, 5, 3, device="cpu").numpy()
    np.testing.assert_array_equal(c, d)
