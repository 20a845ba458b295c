"""The CPU oracle against golden streams written by the reference kernel
itself (tests/golden/ref_golden.npz, made on a B200 by make_ref_golden.py
from PabloEnfedaque/CUDA_BPC-PaCo source/BPC_PaCo.cu built for sm_100a):
every slot word identical, and the oracle decodes them losslessly."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, lut_folder

GOLD = np.load(os.path.join(GOLDEN, "ref_golden.npz"))
CASES = sorted({k.split("/")[0] for k in GOLD.files})


def ref_stream(name, passes, shape):
    n = GOLD[f"{name}/p{passes}/count"]
    words = GOLD[f"{name}/p{passes}/words"]
    out = np.full(shape[0] * shape[1], -1, np.int32).reshape(-1, 4096)
    pos = 0
    for k, c in enumerate(n):
        out[k, :1 + c] = words[pos:pos + 1 + c]
        pos += 1 + c
    assert pos == words.size
    return out.reshape(-1)


@pytest.mark.parametrize("passes", [2, 3])
@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_golden(oracle_mod, luts, name, passes):
    img = GOLD[f"{name}/input"].astype(np.int32)
    want = ref_stream(name, passes, img.shape)
    got = oracle_mod.encode(img, luts(passes), passes)
    bad = np.nonzero(got != want)[0]
    assert bad.size == 0, f"first mismatch at word {bad[:4]}"
    dec = oracle_mod.decode(want, img.shape, luts(passes), passes)
    np.testing.assert_array_equal(dec, img)


def test_golden_covers_edge_cases():
    zero = GOLD["mixed512_zero/input"]
    assert (ref_stream("mixed512_zero", 3, zero.shape).reshape(-1, 4096)[:, 0] == 32).any()
    lap = ref_stream("laplace256_p15", 2, (256, 256)).reshape(-1, 4096)
    assert lap[0, 0] == 15
