"""The autotuner's staged search, on the CPU with a fake timer (the device timing
itself is exercised by tests/test_gpu_autotune.py)."""
import numpy as np
import pytest

from gpu_optical_photons_b200 import autotune
from gpu_optical_photons_b200.params import TallyConfig
from gpu_optical_photons_b200.wavefront import WaveConfig

TALLY = np.arange(12, dtype=np.uint64).reshape(2, 6)


def fake_timer(cost, tallies=lambda cfg: TALLY):
    seen = []

    def time_config(cfg, events, counts, tally, repeats=3, first_id=0):
        seen.append(cfg)
        return cost(cfg), tallies(cfg), {"simt_efficiency": 0.9, "launches": 1}
    return time_config, seen


def test_staged_search_picks_the_fastest_point(monkeypatch):
    # Fastest: 4 blocks/SM, threshold 24, 128-thread blocks, chunk 1024, one wave.
    def cost(c):
        return (abs(c.blocks_per_sm - 4) + abs(c.threshold - 24) / 4 + (c.block_size != 128)
                + (c.cadence != 0) + ((c.chunk or 256) != 1024) + ((c.tail_steps or 4096) != 4096)
                + (c.wave_quota != 0) + 1.0)
    tc, seen = fake_timer(cost)
    monkeypatch.setattr(autotune, "time_config", tc)
    best, log = autotune.tune([None, None], np.array([10, 20]), TallyConfig(), base=WaveConfig())
    assert (best.blocks_per_sm, best.threshold, best.block_size, best.cadence, best.chunk) == \
        (4, 24, 128, 0, 1024)
    assert len(log) == len(seen) and min(r["ms"] for r in log) == cost(best)
    # the first stage covers the full (blocks/SM x threshold) grid
    assert {(c.blocks_per_sm, c.threshold) for c in seen[:20]} == \
        {(b, t) for b in (2, 3, 4, 7) for t in (16, 20, 24, 28, 32)}


def test_seven_blocks_keeps_its_block_size(monkeypatch):
    tc, seen = fake_timer(lambda c: 1.0 if c.blocks_per_sm == 7 else 2.0)
    monkeypatch.setattr(autotune, "time_config", tc)
    best, _ = autotune.tune([None], np.array([5]), TallyConfig(), base=WaveConfig())
    assert best.blocks_per_sm == 7
    # no block-size stage around a 7-blocks point (it implies 128-thread blocks)
    assert all(c.block_size == WaveConfig().block_size for c in seen)


def test_a_setting_that_changes_the_tallies_is_an_error(monkeypatch):
    bad = TALLY.copy()
    bad[0, 0] += 1
    tc, _ = fake_timer(lambda c: 1.0, tallies=lambda c: bad if c.threshold == 20 else TALLY)
    monkeypatch.setattr(autotune, "time_config", tc)
    with pytest.raises(AssertionError):
        autotune.tune([None], np.array([5]), TallyConfig(), base=WaveConfig())
