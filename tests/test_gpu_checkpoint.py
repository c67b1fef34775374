"""Checkpoint and resume of a batched run (optx_engine_run_tally_range,
optx_engine_set_tallies): a batch run as consecutive photon ranges, or stopped
after a checkpoint and resumed by another engine, gives the tallies of one
uninterrupted run exactly (integer sums of histories that depend only on
(seed, photon id)); in exact mode those equal the oracle's."""
import numpy as np
import pytest

from gpu_optical_photons_b200 import params as P
from gpu_optical_photons_b200.wavefront import (WaveConfig, WavefrontEngine, batched_events,
                                                run_tally_checkpointed)

pytestmark = pytest.mark.gpu

TC = P.TallyConfig(100, 50.0, 10)


def make(events, counts, math="fast", first_id=0):
    eng = WavefrontEngine(TC, len(events), int(counts.sum()), WaveConfig(math=math))
    eng.set_events(events, counts, first_id)
    return eng


def test_ranges_equal_one_run(engine):
    events, counts = batched_events(n_events=64, seed=11, median=5000)
    n = int(counts.sum())
    eng = make(events, counts)
    try:
        eng.run_tally()
        whole = eng.tallies()
        # Uneven ranges, cutting through events, including an empty one.
        cuts = [0, 1, 777, n // 3, n // 3, n - 5, n]
        for i, (lo, hi) in enumerate(zip(cuts[:-1], cuts[1:])):
            eng.run_tally_range(lo, hi, accumulate=i > 0)
        assert np.array_equal(eng.tallies(), whole)
        # A plain run afterwards covers the whole batch again and resets the tallies.
        eng.run_tally()
        assert np.array_equal(eng.tallies(), whole)
        # accumulate=False zeroes first: one range gives only its own photons.
        eng.run_tally_range(0, 777, accumulate=False)
        part = eng.tallies()
        assert int(part[:, :5].sum()) == 777
    finally:
        eng.close()


def test_interrupted_run_resumes_exactly(engine, oracle, tmp_path):
    events, counts = batched_events(n_events=48, seed=13, median=3000)
    path = str(tmp_path / "ckpt.npz")
    a = make(events, counts, "exact", first_id=500)
    try:
        _, nxt = run_tally_checkpointed(a, events, counts, 500, path, slice_photons=40_000, stop_after=2)
        assert nxt == 80_000
    finally:
        a.close()  # the process that took the checkpoint is gone
    b = make(events, counts, "exact", first_id=500)
    try:
        got, nxt = run_tally_checkpointed(b, events, counts, 500, path, slice_photons=40_000)
        assert nxt == int(counts.sum())
    finally:
        b.close()
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64) + np.uint64(500)
    arr = (P.CSimParams * len(events))(*[e.to_c() for e in events])
    assert np.array_equal(got, oracle.batch_tally(arr, offs, TC, mode=oracle.PORTABLE))


def test_checkpoint_of_another_batch_is_refused(engine, tmp_path):
    events, counts = batched_events(n_events=16, seed=17, median=2000)
    path = str(tmp_path / "ckpt.npz")
    a = make(events, counts)
    try:
        run_tally_checkpointed(a, events, counts, 0, path, slice_photons=10_000, stop_after=1)
        counts2 = counts.copy()
        counts2[0] += 1
        with pytest.raises(ValueError, match="another batch"):
            run_tally_checkpointed(a, events, counts2, 0, path)
        with pytest.raises(ValueError, match="another batch"):
            run_tally_checkpointed(a, events, counts, 1, path)  # other first_id
    finally:
        a.close()


def test_range_arguments_are_checked(engine):
    events, counts = batched_events(n_events=8, seed=19, median=1000)
    n = int(counts.sum())
    eng = make(events, counts)
    try:
        with pytest.raises(ValueError):
            eng.run_tally_range(10, 5)
        with pytest.raises(ValueError):
            eng.run_tally_range(0, n + 1)
        with pytest.raises(ValueError):
            eng.set_tallies(np.zeros((len(events) + 1, TC.length), np.uint64))
        eng.run_tally()
        whole = eng.tallies()
        eng.run_tally_range(n, n, accumulate=True)  # empty range: tallies unchanged
        assert np.array_equal(eng.tallies(), whole)
        eng.set_tallies(np.zeros_like(whole))
        eng.run_tally_range(0, n, accumulate=True)
        assert np.array_equal(eng.tallies(), whole)
    finally:
        eng.close()
