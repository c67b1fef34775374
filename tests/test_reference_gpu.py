"""This repository's kernels against the reference's own GPU kernels on the same B200.

oracle/relink.py builds the reference's src/gpu/gpu_backend.cu and gpu_event.cu
from its sources for sm_100a (oracle/_ref/libref_gpu*.so). Portable flavour
(OPTPHOT_PORTABLE_MATH, --fmad=false) against EXACT mode: records bit for bit,
tallies equal. Default flavour (CUDA libm, FMA) against FAST mode: the same
fates for >= 99.9 % of photons (the bitwise fraction is printed; both are CUDA
builds of the same expressions, but contraction choices may differ).
"""
import numpy as np
import pytest

from gpu_optical_photons_b200 import params as P
from helpers import compare_histories

pytestmark = pytest.mark.gpu

SETUPS = {
    "default_scat_volume": P.SimParams(scat_length=300.0, source=P.VOLUME),
    "config2": P.config2()[0],
    "config3_all_specular": P.config3(False)[0],
}


def _need(oracle, mode):
    if not oracle.refgpu_available(mode):
        pytest.skip("reference GPU backend not built (python oracle/relink.py needs the reference checkout)")


@pytest.mark.parametrize("setup", list(SETUPS))
def test_records_bitwise_equal_reference_gpu_portable(engine, oracle, setup):
    _need(oracle, oracle.PORTABLE)
    p = SETUPS[setup]
    n = 1_000_000
    ref, _ = oracle.refgpu_records(p, n, first_id=17, mode=oracle.PORTABLE)
    ours, _ = engine.run_gpu_records(p, n, first_id=17, math="exact")
    assert compare_histories(ref, ours)["bitwise_identical"] == n


def test_event_records_bitwise_equal_reference_gpu_portable(engine, oracle):
    _need(oracle, oracle.PORTABLE)
    p = SETUPS["default_scat_volume"]
    n = 300_003
    ref, rst, _ = oracle.refgpu_records_event(p, n, 3, mode=oracle.PORTABLE, chunk=70_001)
    ours, st, _ = engine.run_gpu_records_event(p, n, 3, 256, 0, 70_001, math="exact")
    assert compare_histories(ref, ours)["bitwise_identical"] == n
    assert st["useful_lane_steps"] == rst["useful_lane_steps"]


@pytest.mark.parametrize("setup", list(SETUPS))
def test_tally_equals_reference_gpu_portable(engine, oracle, setup):
    _need(oracle, oracle.PORTABLE)
    p = SETUPS[setup]
    c = P.TallyConfig(500, 50.0, 50)
    n = 2_000_000
    ref, _ = oracle.refgpu_tally(p, c, n, first_id=3, mode=oracle.PORTABLE)
    _, ours, _ = engine.run_gpu_tally(p, c, n, first_id=3, math="exact")
    assert np.array_equal(ref, ours)


@pytest.mark.parametrize("setup", list(SETUPS))
def test_fast_mode_agrees_with_reference_gpu(engine, oracle, setup):
    _need(oracle, oracle.PLATFORM)
    p = SETUPS[setup]
    n = 1_000_000
    ref, _ = oracle.refgpu_records(p, n, mode=oracle.PLATFORM)
    ours, _ = engine.run_gpu_records(p, n, math="fast")
    h = compare_histories(ref, ours)
    print(f"{setup}: bitwise {h['bitwise_identical'] / n:.6f}, same discrete {h['same_discrete'] / n:.6f}, "
          f"fate differs {h['fate_differs']}")
    assert h["fate_differs"] <= 0.001 * n
    assert h["same_discrete"] >= 0.999 * n
