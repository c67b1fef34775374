"""Failure detection without a GPU fault.

Faults are injected on the host (OPTX_TEST_FAULT, read by liboptx at each
call): an allocation that fails as cudaMalloc does when the device is out of
memory, and a wavefront run capped at one wave so that it ends through the
device-side watchdog (the control block's error word, read back by the host).
Neither traps, faults nor hangs the GPU; after each, the same process runs the
same work correctly. Invalid inputs are rejected on the host before any launch.
"""
import numpy as np
import pytest

from gpu_optical_photons_b200 import params as P
from gpu_optical_photons_b200._lib import InvalidArgument, OptxError
from gpu_optical_photons_b200.wavefront import WaveConfig, WavefrontEngine

pytestmark = pytest.mark.gpu

OPTX_ERR_CUDA, OPTX_ERR_WATCHDOG = 3, 6


def test_injected_allocation_failure(engine, monkeypatch):
    monkeypatch.setenv("OPTX_TEST_FAULT", "alloc")
    with pytest.raises(OptxError) as e:
        WavefrontEngine(P.TallyConfig(), 4, 100_000)
    assert e.value.code == OPTX_ERR_CUDA and "out of memory" in str(e.value)
    monkeypatch.delenv("OPTX_TEST_FAULT")
    eng = WavefrontEngine(P.TallyConfig(), 4, 100_000)
    eng.set_events([P.SimParams()], [1000])
    eng.run_tally()
    assert int(eng.tallies()[0, :5].sum()) == 1000
    eng.close()


def test_watchdog_ends_the_run_and_the_engine_recovers(engine, monkeypatch):
    p, c = P.config2()
    n = 200_000
    eng = WavefrontEngine(c, 1, n, WaveConfig(cadence=2, math="exact"))  # needs many waves
    eng.set_events([p], [n])
    monkeypatch.setenv("OPTX_TEST_FAULT", "watchdog")
    eng.run_tally()
    with pytest.raises(OptxError) as e:
        eng.tallies()
    assert e.value.code == OPTX_ERR_WATCHDOG
    monkeypatch.delenv("OPTX_TEST_FAULT")
    eng.run_tally()  # the next run resets the control block
    got = eng.tallies()[0]
    # The one-shot host-buffer calls read the error word in their single wait.
    monkeypatch.setenv("OPTX_TEST_FAULT", "watchdog")
    with pytest.raises(OptxError) as e:
        eng.run_batch([p], [n])
    assert e.value.code == OPTX_ERR_WATCHDOG
    monkeypatch.delenv("OPTX_TEST_FAULT")
    out, st, _ = eng.run_batch([p], [n])
    eng.close()
    _, ref, _ = engine.run_gpu_tally(p, c, n, math="exact")
    assert np.array_equal(got, ref)
    assert np.array_equal(out[0], ref)
    assert st["launches"] > 1 and st["useful_lane_steps"] == int(ref[-2] + ref[-1] + ref[1])


@pytest.mark.parametrize("bad", [
    {"threshold": 33}, {"block_size": 96 + 1}, {"block_size": 512}, {"chunk": 8},
    {"blocks_per_sm": 5}, {"blocks_per_sm": 7, "block_size": 64}])
def test_invalid_engine_settings_rejected(engine, bad):
    with pytest.raises(InvalidArgument):
        WavefrontEngine(P.TallyConfig(), 1, 1000, WaveConfig(**bad))


def test_invalid_parameters_rejected_before_launch(engine):
    for p in (P.SimParams(hx=-1.0), P.SimParams(n_scint=0.0), P.SimParams(abs_length=0.0),
              P.SimParams(tau=-1.0), P.SimParams(surface=7), P.SimParams(source=2)):
        with pytest.raises(InvalidArgument):
            engine.run_gpu_tally(p, P.TallyConfig(), 100)
    # and the device keeps working
    _, flat, _ = engine.run_gpu_tally(P.SimParams(), P.TallyConfig(), 1000)
    assert flat[:5].sum() == 1000


def test_watchdog_in_adjoint_and_score_moment_runs_is_reported(engine, monkeypatch):
    """The replay paths check the run's error word too: a watchdog stop raises
    instead of returning a partial gradient or Jacobian."""
    import torch
    from gpu_optical_photons_b200.adjoint import ResponseModel
    theta = (1000.0, 700.0, 0.95, 4.0)
    tc = P.TallyConfig(500, 50.0, 1)
    m = ResponseModel(P.config2()[0], 200_000, tc, config=WaveConfig(cadence=2))  # many waves
    try:
        w = torch.ones(tc.time_bins + 1, dtype=torch.float64)
        monkeypatch.setenv("OPTX_TEST_FAULT", "watchdog")
        for run in (lambda: m.replay(theta, w, 0.5), lambda: m.score_moments(theta)):
            with pytest.raises(OptxError) as e:
                run()
            assert e.value.code == OPTX_ERR_WATCHDOG
        monkeypatch.delenv("OPTX_TEST_FAULT")
        g = m.replay(theta, w, 0.5)   # the next runs complete
        h, _ = m.score_moments(theta)
        assert np.all(np.isfinite(g)) and h.sum() > 0
    finally:
        m.close()


def test_watchdog_in_records_host_call_is_reported(engine, monkeypatch):
    p = P.config2()[0]
    n = 300_000
    monkeypatch.setenv("OPTX_TEST_FAULT", "watchdog")
    with pytest.raises(OptxError) as e:
        engine.run_gpu_records(p, n)
    assert e.value.code == OPTX_ERR_WATCHDOG
    monkeypatch.delenv("OPTX_TEST_FAULT")
    rec, _ = engine.run_gpu_records(p, n, math="exact")  # the same call completes afterwards
    ref = engine.records_to_numpy(engine.records_device(p, n, math="exact"))
    for k in ("fate", "n_boundary", "n_scatter", "t", "path"):
        assert np.array_equal(rec[k], ref[k]), k


def test_rejected_batch_leaves_the_current_batch_intact(engine):
    """A set_events call that fails on its third event changes nothing: the
    engine still runs the batch uploaded before it."""
    tc = P.TallyConfig(100, 50.0, 10)
    good = [P.config2()[0].replace(abs_length=500.0 + 100.0 * i, max_steps=50 + i) for i in range(4)]
    eng = WavefrontEngine(tc, 4, 40_000)
    try:
        eng.set_events(good, [10_000] * 4)
        eng.run_tally()
        before = eng.tallies()
        bad = [good[3], good[2], P.config2()[0].replace(hx=-1.0), good[0]]
        with pytest.raises(InvalidArgument):
            eng.set_events(bad, [10_000] * 4)
        eng.run_tally()
        assert np.array_equal(eng.tallies(), before)
    finally:
        eng.close()
