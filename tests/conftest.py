"""Shared test helpers.  `-m gpu` tests need a B200; everything else runs on CPU."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "cuda_bpc-paco_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
LUTS = os.path.join(GOLDEN, "luts")
# the reference checkout (BPC_REFERENCE_DIR); only read by CPU tests, which skip without it
REF_ROOT = os.environ.get("BPC_REFERENCE_DIR", "/root/reference")

for p in (PKG, os.path.join(ROOT, "oracle"), GOLDEN):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def lut_folder(passes: int) -> str:
    return os.path.join(LUTS, f"{passes}_coding_pass") + "/"


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def luts(oracle_mod):
    """Loader arrays (oracle) for (passes, levels)."""
    cache = {}

    def get(passes: int, levels: int = 5) -> np.ndarray:
        k = (passes, levels)
        if k not in cache:
            cache[k] = oracle_mod.load_luts(lut_folder(passes), passes, levels)
        return cache[k]

    return get


@pytest.fixture(scope="session")
def sample_subset():
    import make_fixtures
    return make_fixtures.sample_image_from_subset()


@pytest.fixture(scope="session")
def bpc():
    import bpc_paco
    return bpc_paco


def have_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
