"""Per-interaction sorted kernels (optx_sorted_*) against the history kernel and
the reference's golden outputs: records bit for bit, tallies exactly, and the
queue counters against the photons' own step counts."""
import ctypes

import numpy as np
import pytest

from gpu_optical_photons_b200 import _lib, params as P
from gpu_optical_photons_b200._lib import InvalidArgument, OptxError
from gpu_optical_photons_b200.backend import device_records, records_device, records_to_numpy, tally_device
from gpu_optical_photons_b200.wavefront import SortedEngine
from helpers import compare_histories, golden_records, params_from_meta

pytestmark = pytest.mark.gpu

OPTX_ERR_WATCHDOG = 6

GOLDEN_CASES = ["default", "default_scat300_volume", "config1", "config2", "config3_all_specular",
                "black_box", "absorption", "mirror_box", "capped", "big_seed_id"]


def _sorted_records(p, n, first_id=0, math="fast", capacity=0, drain_below=0):
    eng = SortedEngine(capacity, drain_below, math)
    out = device_records(n)
    eng.run(p, n, first_id, records_out=out)
    st = eng.stats()
    eng.close()
    return records_to_numpy(out), st


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_exact_mode_bitwise_equals_reference_portable_build(engine, golden, name):
    """Small queues (many iterations, refills and drains): still the reference's
    portable CPU build bit for bit."""
    arrays, meta = golden
    case = meta["cases"][name]
    p = params_from_meta(case["params"])
    rec, _ = _sorted_records(p, case["n"], case["first_id"], "exact", capacity=1024)
    h = compare_histories(rec, golden_records(arrays, name, "portable"))
    assert h["bitwise_identical"] == case["n"], h


MIXED_FACES = P.SimParams(scat_length=600.0, source=P.VOLUME,
                          face_surface=[P.LAMBERTIAN, P.POLISHED, P.SPECULAR, P.BLACK, P.LAMBERTIAN, 0],
                          face_reflectivity=[0.9, 0.95, 0.97, 0.5, 0.85, 0.0])


def _setup(cfg):
    if cfg == "config3_ref":
        return P.config3(black_minus_z=False)[0]
    if cfg == "mixed_faces":  # every face model, photons moving between all three queues
        return MIXED_FACES
    return getattr(P, cfg)()[0]


@pytest.mark.parametrize("cfg", ["config1", "config2", "config3", "config3_ref", "mixed_faces"])
@pytest.mark.parametrize("math_mode", ["fast", "exact", "approx"])
def test_records_equal_history_kernel(engine, cfg, math_mode):
    p = _setup(cfg)
    n = 300_001  # not a multiple of 32
    hist = records_to_numpy(records_device(p, n, first_id=7, math=math_mode))
    for cap, drain in ((0, 0), (4096, 1), (8192, 3000)):
        rec, st = _sorted_records(p, n, 7, math_mode, cap, drain)
        h = compare_histories(rec, hist)
        assert h["bitwise_identical"] == n, (cap, drain, h)


@pytest.mark.parametrize("cfg", ["config1", "config2", "config3", "mixed_faces"])
def test_tally_equals_history_tally(engine, cfg):
    p, c = (MIXED_FACES, P.TallyConfig(200, 50.0, 20)) if cfg == "mixed_faces" else getattr(P, cfg)()
    n = 1_000_000
    ref = tally_device(p, c, n).cpu().numpy()
    eng = SortedEngine(1 << 16)
    got, _ = eng.run(p, n, tally=c)
    got = got.cpu().numpy()
    assert np.array_equal(got, ref)
    eng.close()


def test_tally_accumulates_and_records_in_one_run(engine):
    import torch
    p, c = P.config2()
    n = 200_000
    ref = tally_device(p, c, n, first_id=5).cpu().numpy()
    eng = SortedEngine(1 << 14)
    t = torch.zeros(c.length, dtype=torch.int64, device="cuda")
    out = device_records(n)
    eng.run(p, n, 5, tally=c, tally_out=t, records_out=out)
    eng.run(p, n, 5, tally=c, tally_out=t)
    eng.close()
    assert np.array_equal(t.cpu().numpy(), 2 * ref)
    hist = records_to_numpy(records_device(p, n, first_id=5))
    assert compare_histories(records_to_numpy(out), hist)["bitwise_identical"] == n


def test_queue_counters_match_the_photons_steps(engine):
    """With no drain, every step after emission goes through a queue: the scatter
    queue saw sum(n_scatter) photons, the face queues sum(n_boundary) (no black
    faces here), and the run took as many iterations as the longest history
    plus the emission one."""
    p = P.config2()[0]
    n = 100_000
    rec, st = _sorted_records(p, n, 0, "fast", capacity=1 << 17, drain_below=1)
    assert st["drained"] == 0
    assert st["queued"]["scatter"] == int(rec["n_scatter"].astype(np.int64).sum())
    assert st["queued"]["polished"] + st["queued"]["painted"] == int(rec["n_boundary"].astype(np.int64).sum())
    longest = int((rec["n_scatter"].astype(np.int64) + rec["n_boundary"]).max())
    assert st["iterations"] == longest + 1
    # The same run with the default drain finishes in fewer launches, same records.
    rec2, st2 = _sorted_records(p, n, 0, "fast", capacity=1 << 17)
    assert st2["drained"] == n and st2["iterations"] == 1
    assert compare_histories(rec2, rec)["bitwise_identical"] == n


def test_step_limit_and_black_faces(engine):
    p = P.config3()[0]  # black -z face
    p.max_steps = 5
    n = 50_000
    hist = records_to_numpy(records_device(p, n, math="exact"))
    rec, st = _sorted_records(p, n, 0, "exact", capacity=2048, drain_below=1)
    assert compare_histories(rec, hist)["bitwise_identical"] == n
    assert (rec["fate"] == P.MAX_STEPS).sum() > 0
    assert (rec["fate"] == P.ABSORBED_SURFACE).sum() > 0


def test_single_photon_and_invalid_arguments(engine):
    p = P.config1()[0]
    rec, st = _sorted_records(p, 1, 123)
    hist = records_to_numpy(records_device(p, 1, first_id=123))
    assert compare_histories(rec, hist)["bitwise_identical"] == 1
    eng = SortedEngine()
    with pytest.raises(InvalidArgument):
        eng.run(p, 10)  # neither a tally nor records
    with pytest.raises(InvalidArgument):
        eng.run(p, 1 << 32, tally=P.config1()[1])
    eng.close()
    with pytest.raises(InvalidArgument):
        SortedEngine(capacity=(1 << 28) + 64)


def test_watchdog_ends_the_run_and_the_next_run_recovers(engine, monkeypatch):
    p, c = P.config2()
    n = 100_000
    eng = SortedEngine(4096)
    monkeypatch.setenv("OPTX_TEST_FAULT", "watchdog")
    eng.run(p, n, tally=c)
    with pytest.raises(OptxError) as e:
        eng.stats()
    assert e.value.code == OPTX_ERR_WATCHDOG
    monkeypatch.delenv("OPTX_TEST_FAULT")
    got, _ = eng.run(p, n, tally=c)
    eng.stats()
    eng.close()
    assert np.array_equal(got.cpu().numpy(), tally_device(p, c, n).cpu().numpy())


def test_host_loop_runs_the_same_iterations(engine):
    """OPTX_SORTED_HOST_LOOP (host-launched iterations, for profilers) gives the
    graph loop's records and iteration count."""
    p = P.config2()[0]
    n = 300_000
    recs, its = [], []
    for host_loop in (False, True):
        eng = SortedEngine(1 << 15, 0, "fast", host_loop=host_loop)
        out = device_records(n)
        eng.run(p, n, records_out=out)
        its.append(eng.stats()["iterations"])
        eng.close()
        recs.append(records_to_numpy(out))
    assert its[0] == its[1] > 8
    assert compare_histories(recs[0], recs[1])["bitwise_identical"] == n
    h = ctypes.c_void_p()
    with pytest.raises(InvalidArgument):
        _lib.call("optx_sorted_create", ctypes.byref(_lib.CSortedConfig(0, 0, 0, 0, 2)), ctypes.byref(h))
    with pytest.raises(InvalidArgument):
        SortedEngine(blocks_per_sm=5)


def test_output_buffers_are_checked_before_launch(engine):
    import torch
    p, c = P.config1()
    eng = SortedEngine(4096)
    with pytest.raises(ValueError):
        eng.run(p, 1000, tally=c, tally_out=torch.zeros(c.length - 1, dtype=torch.int64, device="cuda"))
    with pytest.raises(ValueError):
        eng.run(p, 1000, tally=c, tally_out=torch.zeros(c.length, dtype=torch.int32, device="cuda"))
    with pytest.raises(ValueError):
        eng.run(p, 1000, records_out=device_records(999))
    out, _ = eng.run(p, 1000, tally=c)  # the engine is untouched by the refusals
    eng.stats()
    eng.close()
    assert int(out[:5].sum()) == 1000


def test_history_and_engine_wrappers_check_their_buffers(engine):
    import torch
    from gpu_optical_photons_b200.wavefront import WavefrontEngine
    p, c = P.config1()
    with pytest.raises(ValueError):
        records_device(p, 100, out=device_records(99))
    with pytest.raises(ValueError):
        tally_device(p, c, 100, out=torch.zeros(c.length, dtype=torch.int64))  # host tensor
    eng = WavefrontEngine(c, 1, 1000)
    eng.set_events([p], [1000])
    with pytest.raises(ValueError):
        eng.run_records(device_records(999))
    out = device_records(1000)
    eng.run_records(out)
    eng.close()
    assert compare_histories(records_to_numpy(out), records_to_numpy(records_device(p, 1000)))["bitwise_identical"] == 1000


def test_sorted_autotuner_picks_a_measured_setting(engine):
    from gpu_optical_photons_b200.autotune import tune_sorted
    p, c = P.config2()
    n = 2_000_000
    best, table = tune_sorted(p, c, n, capacities=(1 << 16, 1 << 18), repeats=2)
    assert set(table) == {(b, k) for b in (3, 4) for k in (1 << 16, 1 << 18)}
    assert table[(best["blocks_per_sm"], best["capacity"])] == min(table.values())
    eng = SortedEngine(best["capacity"], blocks_per_sm=best["blocks_per_sm"])
    got, _ = eng.run(p, n, tally=c)
    eng.stats()
    eng.close()
    assert np.array_equal(got.cpu().numpy(), tally_device(p, c, n).cpu().numpy())
