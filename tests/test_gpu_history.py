"""History (plain) kernel through the C ABI against the oracle and the reference's
golden outputs. Modelled on the reference's tests/test_gpu.cpp."""
import math

import numpy as np
import pytest

from gpu_optical_photons_b200 import params as P
from helpers import (binomial_pull, chi2_two_sample, compare_histories, face_solid_angle_fraction,
                     face_survival_fraction, golden_records, ks_two_sample, params_from_meta,
                     steps_of)

pytestmark = pytest.mark.gpu

GOLDEN_CASES = ["default", "default_scat300_volume", "config1", "config2", "config3_all_specular",
                "black_box", "absorption", "mirror_box", "capped", "big_seed_id"]


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_exact_mode_bitwise_equals_reference_portable_build(engine, golden, name):
    """Exact mode (portable math, no FMA) = the reference's OPTPHOT_PORTABLE_MATH CPU build, bit for bit."""
    arrays, meta = golden
    case = meta["cases"][name]
    p = params_from_meta(case["params"])
    rec, _ = engine.run_gpu_records(p, case["n"], first_id=case["first_id"], math="exact")
    h = compare_histories(rec, golden_records(arrays, name, "portable"))
    assert h["bitwise_identical"] == case["n"], h


@pytest.mark.parametrize("name", GOLDEN_CASES)
@pytest.mark.parametrize("math_mode", ["fast", "approx"])
def test_fast_mode_agrees_with_reference_default_build(engine, golden, name, math_mode):
    arrays, meta = golden
    case = meta["cases"][name]
    p = params_from_meta(case["params"])
    rec, _ = engine.run_gpu_records(p, case["n"], first_id=case["first_id"], math=math_mode)
    h = compare_histories(rec, golden_records(arrays, name, "platform"))
    # Tolerance: at most 0.1% of histories with a different discrete path.
    assert h["same_discrete"] >= 0.999 * case["n"] - 1, h


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


@pytest.mark.parametrize("name", list(PARITY))
def test_exact_mode_bitwise_equals_oracle(engine, oracle, name):
    p = PARITY[name]
    n = 200_000
    rec, _ = engine.run_gpu_records(p, n, first_id=77, math="exact")
    ref = oracle.records(p, n, 77, mode=oracle.PORTABLE)
    h = compare_histories(rec, ref)
    assert h["bitwise_identical"] == n, h


@pytest.mark.parametrize("name", list(PARITY))
@pytest.mark.parametrize("math_mode", ["fast", "approx"])
def test_fast_mode_fate_agreement(engine, oracle, name, math_mode):
    """>= 99.9% of photons with the same fate and step counts as the CPU FP32 run."""
    p = PARITY[name]
    n = 1_000_000
    rec, _ = engine.run_gpu_records(p, n, math=math_mode)
    ref = oracle.records(p, n, 0, mode=oracle.PLATFORM)
    h = compare_histories(rec, ref)
    assert h["fate_differs"] <= 0.001 * n, h
    assert h["same_discrete"] >= 0.999 * n, h


@pytest.mark.parametrize("name", ["config1", "config2", "config3_black_minus_z"])
@pytest.mark.parametrize("math_mode", ["exact", "fast"])
def test_tally_matches_oracle(engine, oracle, name, math_mode):
    p = PARITY[name]
    c = P.TallyConfig(500, 50.0, 50)
    n = 300_000
    t, flat, _ = engine.run_gpu_tally(p, c, n, math=math_mode)
    ref = oracle.tally(p, c, n, 0, mode=oracle.PORTABLE if math_mode == "exact" else oracle.PLATFORM)
    if math_mode == "exact":
        assert np.array_equal(flat, ref)  # integer tallies exact
    else:
        assert t.total() == n
        chi2, ndf, pv = chi2_two_sample(flat[5:5 + 501], ref[5:5 + 501])
        assert pv > 0.01, (chi2, ndf)
        assert abs(int(flat[0]) - int(ref[0])) <= 0.001 * n


def test_tally_agrees_with_records_and_block_size(engine):
    """tests/test_gpu.cpp:122-146: tally == records; bit-identical across block sizes."""
    p = P.SimParams()
    c = P.TallyConfig()
    n = 1_000_000
    rec, _ = engine.run_gpu_records(p, n)
    t1, f1, _ = engine.run_gpu_tally(p, c, n)
    t2, f2, _ = engine.run_gpu_tally(p, c, n, block_size=128)
    t3, f3, _ = engine.run_gpu_tally(p, c, n, block_size=512)
    assert np.array_equal(t1.fate_counts, np.bincount(rec["fate"], minlength=5))
    assert np.array_equal(f1, f2) and np.array_equal(f1, f3)
    assert t1.boundary_sum == int(rec["n_boundary"].sum())
    assert t1.scatter_sum == int(rec["n_scatter"].sum())
    assert t1.time_hist.sum() == t1.fate_counts[0]


def test_records_independent_of_chunk_and_block(engine):
    """tests/test_gpu.cpp:148-158."""
    p = P.SimParams(scat_length=300.0)
    n = 300_000
    a, _ = engine.run_gpu_records(p, n, 256, 0, 1 << 24)
    b, _ = engine.run_gpu_records(p, n, 64, 0, 70001)
    assert compare_histories(a, b)["bitwise_identical"] == n


def test_first_id_offsets(engine):
    p = P.SimParams(scat_length=300.0)
    a, _ = engine.run_gpu_records(p, 10_000, first_id=0)
    b, _ = engine.run_gpu_records(p, 500, first_id=1000)
    assert compare_histories({k: v[1000:1500] for k, v in a.items()}, b)["bitwise_identical"] == 500


def test_independent_seeds_statistically_compatible(engine, oracle):
    """tests/test_gpu.cpp:102-120: GPU (seed+1) vs CPU (seed): efficiency z, time chi2/KS, hit-map chi2."""
    p = P.SimParams(scat_length=300.0)
    n = 2_000_000
    cpu = oracle.records(p, n, 0)
    gpu, _ = engine.run_gpu_records(p.replace(seed=p.seed + 1), n)
    da, db = cpu["fate"] == 0, gpu["fate"] == 0
    ea, eb = da.mean(), db.mean()
    z = (ea - eb) / math.sqrt(ea * (1 - ea) / n + eb * (1 - eb) / n)
    assert abs(z) < 4
    tmax = np.nextafter(max(cpu["t"][da].max(), gpu["t"][db].max()), np.inf)
    ha = np.histogram(cpu["t"][da], bins=100, range=(0, tmax))[0]
    hb = np.histogram(gpu["t"][db], bins=100, range=(0, tmax))[0]
    assert chi2_two_sample(ha, hb)[2] > 1e-4
    assert ks_two_sample(cpu["t"][da], gpu["t"][db])[1] > 1e-4
    xa = np.histogram2d(cpu["x"][da], cpu["y"][da], bins=20, range=[[-25, 25], [-25, 25]])[0].ravel()
    xb = np.histogram2d(gpu["x"][db], gpu["y"][db], bins=20, range=[[-25, 25], [-25, 25]])[0].ravel()
    assert chi2_two_sample(xa, xb)[2] > 1e-4


def test_solid_angle(engine):
    """tests/test_gpu.cpp:50-61: black walls, index-matched readout: P(det) = Omega / 4pi."""
    p = P.black_box().replace(src_x=10.0, src_y=-5.0, src_z=3.0)
    n = 4_000_000
    t, _, _ = engine.run_gpu_tally(p, P.TallyConfig(), n)
    expected = face_solid_angle_fraction(p, 5)
    assert abs(binomial_pull(int(t.fate_counts[0]), n, expected)) < 4


def test_absorption_quadrature(engine):
    """tests/test_gpu.cpp:63-75: absorption L = 100 mm against Gauss-Legendre quadrature."""
    p = P.black_box().replace(src_x=10.0, src_y=-5.0, src_z=3.0, abs_length=100.0)
    n = 4_000_000
    t, _, _ = engine.run_gpu_tally(p, P.TallyConfig(), n)
    expected = face_survival_fraction(p, 5, 100.0)
    assert abs(binomial_pull(int(t.fate_counts[0]), n, expected)) < 4


def test_edge_cases(engine):
    p = P.SimParams()
    rec, _ = engine.run_gpu_records(p, 0)
    assert len(rec) == 0
    t, flat, _ = engine.run_gpu_tally(p, P.TallyConfig(), 0)
    assert flat.sum() == 0
    rec, _ = engine.run_gpu_records(p.replace(max_steps=0), 100)
    assert (rec["fate"] == P.MAX_STEPS).all() and (rec["n_boundary"] == 0).all()
    with pytest.raises(ValueError):
        engine.run_gpu_records(p, 10, block_size=100)
    with pytest.raises(engine.OptxError):
        engine.run_gpu_tally(p, P.TallyConfig(100, 50.0, 300), 10)  # 360 KB of shared-memory bins
    # the failure leaves no CUDA error behind for the next launch
    rec, _ = engine.run_gpu_records(p, 1000)
    assert len(rec) == 1000
    # 223 KB of bins: too many for the wavefront engine beside its pantries, so the
    # host call runs the history kernel, with the same result as the device call
    c = P.TallyConfig(100, 50.0, 236)
    _, flat, _ = engine.run_gpu_tally(p, c, 20_000, first_id=5)
    dev = engine.tally_device(p, c, 20_000, first_id=5)
    assert np.array_equal(flat, dev.cpu().numpy().astype(np.uint64))
    assert flat[:5].sum() == 20_000


def test_records_pipeline_pinned_and_pageable(engine):
    """Multi-chunk records (several pipeline stages) equal one-shot device records, for
    pageable numpy arrays and for pinned arrays (direct DMA)."""
    import torch
    p = P.config2()[0]
    n = 9_000_001  # > 2 pipeline buffer sets of 2^22, ragged last chunk
    d = engine.records_device(p, n, first_id=3)
    torch.cuda.synchronize()
    want = engine.records_to_numpy(d)
    rec, tm = engine.run_gpu_records(p, n, first_id=3)
    assert compare_histories(rec, want)["bitwise_identical"] == n
    pinned = engine.Records()
    for k in engine.Records.FIELDS:
        dt = {"fate": torch.uint8, "n_boundary": torch.int32, "n_scatter": torch.int32}.get(k, torch.float32)
        a = torch.empty(n, dtype=dt, pin_memory=True).numpy()
        pinned[k] = a.view(np.uint32) if k in ("n_boundary", "n_scatter") else a
    rec2, _ = engine.run_gpu_records(p, n, first_id=3, out=pinned)
    assert compare_histories(rec2, want)["bitwise_identical"] == n
    small, _ = engine.run_gpu_records(p, 1000, first_id=3, chunk=77)  # many tiny chunks
    assert compare_histories(small, {k: v[:1000] for k, v in want.items()})["bitwise_identical"] == 1000


def test_host_call_engine_cache_eviction(engine):
    """Host tally calls with more tally configurations than the engine cache holds
    (8), interleaved: every result equals the device history kernel's."""
    p = P.config2()[0]
    for i in range(12):
        c = P.TallyConfig(50 + 7 * i, 50.0, 3 + i % 4)
        _, flat, _ = engine.run_gpu_tally(p, c, 50_000, first_id=i)
        dev = engine.tally_device(p, c, 50_000, first_id=i)
        assert np.array_equal(flat, dev.cpu().numpy().astype(np.uint64)), i
    from gpu_optical_photons_b200 import _lib
    before, _ = engine.run_gpu_records(p, 20_000, first_id=5)
    assert _lib.lib().optx_release_cache() == 0   # engines, staging and pipeline buffers
    _, flat, _ = engine.run_gpu_tally(p, P.TallyConfig(), 10_000)  # a fresh engine after release
    assert flat[:5].sum() == 10_000
    after, _ = engine.run_gpu_records(p, 20_000, first_id=5)  # re-created pipeline buffers
    assert compare_histories(after, before)["bitwise_identical"] == 20_000


def test_host_calls_from_several_threads(engine):
    """Concurrent host calls (tally and records, two tally configurations) from
    four threads give the results of the same calls made one at a time."""
    from concurrent.futures import ThreadPoolExecutor
    p = P.config2()[0]
    cs = [P.TallyConfig(100, 50.0, 10), P.TallyConfig(200, 40.0, 5)]

    def job(i):
        if i % 3 == 2:
            rec, _ = engine.run_gpu_records(p, 40_000, first_id=i)
            return ("rec", i, int(rec["n_boundary"].sum()), int(rec["fate"].astype(np.int64).sum()))
        _, flat, _ = engine.run_gpu_tally(p, cs[i % 2], 60_000, first_id=i)
        return ("tally", i, flat.tobytes())

    serial = [job(i) for i in range(12)]
    with ThreadPoolExecutor(4) as pool:
        parallel = list(pool.map(job, range(12)))
    assert serial == parallel


def test_event_records_and_cache_release_from_several_threads(engine):
    """Event-kernel records calls of growing sizes (so the cached device buffer
    is re-allocated) interleaved with cache releases on four threads give the
    results of the same calls made one at a time."""
    from concurrent.futures import ThreadPoolExecutor
    from gpu_optical_photons_b200 import _lib
    p = P.config2()[0]

    def job(i):
        if i % 4 == 3:
            assert _lib.lib().optx_release_cache() == 0
            return ("release", i)
        n = 20_000 + 15_000 * i
        rec, _, _ = engine.run_gpu_records_event(p, n, 4, first_id=i)
        return ("event", i, int(rec["n_boundary"].sum()), float(rec["t"].astype(np.float64).sum()))

    serial = [job(i) for i in range(12)]
    with ThreadPoolExecutor(4) as pool:
        parallel = list(pool.map(job, range(12)))
    assert serial == parallel
