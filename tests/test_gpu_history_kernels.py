"""The plain history kernels themselves against the oracle and the reference's
golden outputs, through the device calls that launch them and nothing else:
optx_records_device (history_records_kernel, one thread per photon, the drop-in
for the reference's transport_records_kernel, src/gpu/gpu_backend.cu:47-52) and
optx_tally_device (history_tally_kernel, the drop-in for transport_tally_kernel,
gpu_backend.cu:56-100). The host calls optx_run_records / optx_run_tally run the
wavefront engine, so these are the only tests that pin the history kernels
without going through another GPU path. Modelled on the reference's
tests/test_gpu.cpp:77-146."""
import numpy as np
import pytest

from gpu_optical_photons_b200 import params as P
from helpers import (check_tally_consistency, chi2_two_sample, compare_histories, golden_records,
                     params_from_meta)

pytestmark = pytest.mark.gpu

GOLDEN_CASES = ["default", "default_scat300_volume", "config1", "config2", "config3_all_specular",
                "black_box", "absorption", "mirror_box", "capped", "big_seed_id"]

PARITY = {
    "config1": P.config1()[0],
    "config2": P.config2()[0],
    "config3_black_minus_z": P.config3(True)[0],
    "polished_scat_volume": P.SimParams(scat_length=300.0, source=P.VOLUME),
    "specular_faces": P.SimParams(surface=P.SPECULAR, reflectivity=0.9, scat_length=400.0),
    "mixed_faces": P.SimParams(scat_length=600.0, source=P.VOLUME,
                               face_surface=[P.LAMBERTIAN, P.POLISHED, P.SPECULAR, P.BLACK,
                                             P.LAMBERTIAN, 0],
                               face_reflectivity=[0.9, 0.95, 0.97, 0.5, 0.85, 0.0]),
}


def history_records(engine, p, n, first_id, math, block_size=256):
    """history_records_kernel only: optx_records_device into device arrays."""
    import torch
    d = engine.records_device(p, n, first_id=first_id, math=math, block_size=block_size)
    torch.cuda.synchronize()
    return engine.records_to_numpy(d)


def history_tally(engine, p, c, n, first_id, math, block_size=256):
    """history_tally_kernel only: optx_tally_device into a zeroed device tally."""
    t = engine.tally_device(p, c, n, first_id=first_id, math=math, block_size=block_size)
    return t.cpu().numpy().astype(np.uint64)


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_history_records_kernel_exact_bitwise_equals_golden(engine, golden, name):
    """Exact mode = the reference's OPTPHOT_PORTABLE_MATH CPU build, bit for bit."""
    arrays, meta = golden
    case = meta["cases"][name]
    p = params_from_meta(case["params"])
    rec = history_records(engine, p, case["n"], case["first_id"], "exact")
    h = compare_histories(rec, golden_records(arrays, name, "portable"))
    assert h["bitwise_identical"] == case["n"], h


@pytest.mark.parametrize("name", GOLDEN_CASES)
@pytest.mark.parametrize("math_mode", ["fast", "approx"])
def test_history_records_kernel_fast_agrees_with_golden(engine, golden, name, math_mode):
    """Fast / approx = the reference's default CPU build for >= 99.9 % of histories."""
    arrays, meta = golden
    case = meta["cases"][name]
    p = params_from_meta(case["params"])
    rec = history_records(engine, p, case["n"], case["first_id"], math_mode)
    h = compare_histories(rec, golden_records(arrays, name, "platform"))
    assert h["same_discrete"] >= 0.999 * case["n"] - 1, h


@pytest.mark.parametrize("name", list(PARITY))
def test_history_records_kernel_exact_bitwise_equals_oracle(engine, oracle, name):
    p = PARITY[name]
    n = 200_000
    rec = history_records(engine, p, n, 77, "exact")
    h = compare_histories(rec, oracle.records(p, n, 77, mode=oracle.PORTABLE))
    assert h["bitwise_identical"] == n, h


@pytest.mark.parametrize("name", list(PARITY))
def test_history_records_kernel_fast_fate_agreement(engine, oracle, name):
    """>= 99.9 % of photons with the same fate and step counts as the CPU FP32 run,
    <= 0.1 % with a different fate."""
    p = PARITY[name]
    n = 1_000_000
    rec = history_records(engine, p, n, 0, "fast")
    h = compare_histories(rec, oracle.records(p, n, 0, mode=oracle.PLATFORM))
    assert h["fate_differs"] <= 0.001 * n, h
    assert h["same_discrete"] >= 0.999 * n, h


@pytest.mark.parametrize("name", ["config1", "config2", "config3_black_minus_z", "mixed_faces"])
def test_history_tally_kernel_exact_equals_oracle(engine, oracle, name):
    """Integer tallies exactly equal to the oracle's (portable math)."""
    p = PARITY[name]
    c = P.TallyConfig(500, 50.0, 50)
    n = 300_000
    got = history_tally(engine, p, c, n, 11, "exact")
    want = oracle.tally(p, c, n, 11, mode=oracle.PORTABLE)
    assert np.array_equal(got, want)
    check_tally_consistency(got, c)


@pytest.mark.parametrize("name", ["config1", "config2", "config3_black_minus_z"])
def test_history_tally_kernel_fast_matches_oracle_statistically(engine, oracle, name):
    p = PARITY[name]
    c = P.TallyConfig(500, 50.0, 50)
    n = 1_000_000
    got = history_tally(engine, p, c, n, 0, "fast")
    want = oracle.tally(p, c, n, 0, mode=oracle.PLATFORM)
    assert int(got[:5].sum()) == n
    assert abs(int(got[0]) - int(want[0])) <= 0.001 * n
    for lo, hi in ((5, 5 + 501), (5 + 501, 5 + 501 + 2500)):  # arrival times, hit map
        chi2, ndf, pv = chi2_two_sample(got[lo:hi], want[lo:hi])
        assert pv > 0.01, (lo, chi2, ndf)


def test_history_kernels_independent_of_block_size(engine, oracle):
    """tests/test_gpu.cpp:122-158: tallies bit-identical across block sizes, records
    independent of the block size, tally fates = record fates."""
    p = P.SimParams(scat_length=300.0, source=P.VOLUME)
    c = P.TallyConfig()
    n = 500_000
    tallies = [history_tally(engine, p, c, n, 3, "fast", bs) for bs in (64, 128, 256, 512, 1024)]
    for t in tallies[1:]:
        assert np.array_equal(t, tallies[0])
    recs = [history_records(engine, p, n, 3, "fast", bs) for bs in (32, 256, 1024)]
    for r in recs[1:]:
        assert compare_histories(r, recs[0])["bitwise_identical"] == n
    assert np.array_equal(tallies[0][:5], np.bincount(recs[0]["fate"], minlength=5))
    assert int(tallies[0][-2]) == int(recs[0]["n_boundary"].astype(np.int64).sum())
    assert int(tallies[0][-1]) == int(recs[0]["n_scatter"].astype(np.int64).sum())


def test_history_kernels_edge_cases(engine, oracle):
    """Empty runs, max_steps = 0 and a ragged last block reach the kernels' bounds."""
    p = P.config2()[0]
    c = P.TallyConfig(100, 50.0, 10)
    assert history_tally(engine, p, c, 0, 0, "exact").sum() == 0
    capped = p.replace(max_steps=0)
    rec = history_records(engine, capped, 1000, 0, "exact")
    assert (rec["fate"] == P.MAX_STEPS).all() and (rec["n_boundary"] == 0).all()
    n = 256 * 3 + 17  # ragged last block
    rec = history_records(engine, p, n, 5, "exact")
    assert compare_histories(rec, oracle.records(p, n, 5, mode=oracle.PORTABLE))["bitwise_identical"] == n
    assert np.array_equal(history_tally(engine, p, c, n, 5, "exact"),
                          oracle.tally(p, c, n, 5, mode=oracle.PORTABLE))
