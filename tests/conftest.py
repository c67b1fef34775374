"""Shared fixtures. GPU tests are marked `gpu` and call the engine through the
C ABI (liboptx.so); everything else runs on the CPU."""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests through the C ABI")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    if not os.path.exists(O.ORACLE_SO):
        O.build(with_ref=False)
    return O


@pytest.fixture(scope="session")
def golden():
    arrays = np.load(os.path.join(GOLDEN, "golden_records.npz"))
    with open(os.path.join(GOLDEN, "golden_meta.json")) as f:
        meta = json.load(f)
    return arrays, meta


@pytest.fixture(scope="session")
def engine():
    """The package with liboptx.so built and a GPU present (fails loudly otherwise)."""
    from gpu_optical_photons_b200 import build
    build.build()
    import gpu_optical_photons_b200 as g
    assert g.gpu_available(), "a gpu-marked test needs a CUDA device"
    return g
