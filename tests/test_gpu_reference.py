"""The oracle against the reference kernel itself (PabloEnfedaque/CUDA_BPC-PaCo
source/BPC_PaCo.cu rebuilt for sm_100a by oracle/Makefile into oracle/_ref/),
run on the GPU: identical streams, identical decodes.  Skipped where the
reference build is absent."""
import numpy as np
import pytest

import bpc_synth
from conftest import lut_folder

pytestmark = pytest.mark.gpu

ref_run = pytest.importorskip("ref_run")


def need(passes):
    if not ref_run.available(passes):
        pytest.skip("reference kernel not built (make -C oracle ref)")


@pytest.mark.parametrize("passes", [2, 3])
def test_reference_encode_sample_subset(oracle_mod, luts, sample_subset, passes):
    """The sample's codeblocks plus ~900 all-zero codeblocks (MSB = 32)."""
    need(passes)
    lut = luts(passes)
    got = ref_run.ref_encode(sample_subset, lut, passes)
    np.testing.assert_array_equal(got, oracle_mod.encode(sample_subset, lut, passes))


def test_reference_decode_sample_subset_2pass(oracle_mod, luts, sample_subset):
    need(2)
    lut = luts(2)
    s = oracle_mod.encode(sample_subset, lut, 2)
    np.testing.assert_array_equal(ref_run.ref_decode(s, sample_subset.shape, lut, 2), sample_subset)


@pytest.mark.parametrize("passes", [2, 3])
@pytest.mark.parametrize("side,seed", [(512, 5), (2048, 1)])
def test_reference_synthetic(oracle_mod, luts, passes, side, seed):
    need(passes)
    img = bpc_synth.synthetic_coefficients(side, 5, seed, amp=40)
    lut = luts(passes)
    want = oracle_mod.encode(img, lut, passes)
    np.testing.assert_array_equal(ref_run.ref_encode(img, lut, passes), want)
    if passes == 2 or not (want.reshape(-1, 4096)[:, 0] == 32).any():
        np.testing.assert_array_equal(ref_run.ref_decode(want, img.shape, lut, passes), img)


@pytest.mark.parametrize("passes", [2, 3])
def test_reference_laplacian_plane15(oracle_mod, luts, passes):
    """Bitplane 15 populated: the reference reads LUT entries past the
    loader's array (zero-padded allocation here)."""
    need(passes)
    img = bpc_synth.laplacian_coefficients(512, 5, 4)
    img[0, 0] = 40000
    lut = luts(passes)
    want = oracle_mod.encode(img, lut, passes)
    np.testing.assert_array_equal(ref_run.ref_encode(img, lut, passes), want)


@pytest.mark.parametrize("passes", [2, 3])
def test_reference_equals_product(bpc, luts, passes):
    """Product kernel == reference kernel on the same input, directly."""
    need(passes)
    img = bpc_synth.synthetic_coefficients(1024, 5, 12, amp=40)
    lut_np = luts(passes)
    lut = bpc.DeviceLut(lut_folder(passes), passes, 5)
    try:
        ours, st = bpc.encode_host(img, lut)
    finally:
        lut.close()
    assert st == 0
    np.testing.assert_array_equal(ours, ref_run.ref_encode(img, lut_np, passes))
