"""The autotuner on the device: a small sweep over the batched workload returns
settings that run, are among those it timed, and give the default settings'
tallies (the engine's results do not depend on its settings)."""
import numpy as np
import pytest

from gpu_optical_photons_b200.autotune import time_config, tune
from gpu_optical_photons_b200.params import TallyConfig
from gpu_optical_photons_b200.wavefront import WaveConfig, batched_events

pytestmark = pytest.mark.gpu


def test_tune_small_batch(engine):
    events, counts = batched_events(n_events=96, median=2e3)
    tc = TallyConfig(100, 50.0, 10)
    best, log = tune(events, counts, tc, repeats=1, bps=(3, 7), thresholds=(24, 28),
                     blocks=(128,), cadences=(0, 8), quota_fracs=(0.0,), chunks=(64,), tails=(4096,))
    assert len(log) >= 4 + 1 + 1
    assert min(r["ms"] for r in log) > 0
    assert any(all(r[k] == getattr(best, k) for k in ("blocks_per_sm", "threshold", "block_size",
                                                      "cadence", "chunk")) for r in log)
    _, t_best, _ = time_config(best, events, counts, tc, repeats=1)
    _, t_default, _ = time_config(WaveConfig(), events, counts, tc, repeats=1)
    assert np.array_equal(t_best, t_default)
    assert int(t_best[:, :5].sum()) == int(counts.sum())
