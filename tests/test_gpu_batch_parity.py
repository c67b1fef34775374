"""The benchmarked batch itself against the oracle: all 4096 events of the
batched workload (66.5 M photons; lognormal photons per event, per-event
absorption, reflectivity, refractive index and scattering; Lambertian cube;
100 arrival-time bins over 0-50 ns, 10 x 10 hit map), at full size.

* Exact mode: every per-event integer tally equals the oracle's (portable math,
  the reference's OPTPHOT_PORTABLE_MATH CPU build), for the engine settings the
  benchmark runs (7 blocks of 128 threads, the 72-register budget), the default
  settings, and the plain history kernel launched once per event.
* Fast and approx modes: against the oracle's default-math CPU run of the same photons, the
  detected counts differ by <= 1e-3 of the photons, the per-event fate counts by
  <= 1e-3 in total, and the summed arrival-time histogram and hit map pass the
  two-sample chi-squared test (p > 0.01); on the first 64 events the per-photon
  records agree in fate for >= 99.9 % of photons.
Each event owns photon ids offset_i .. offset_i + n_i - 1, so event i is the
reference's run_cpu_tally(p_i, n_i, first_id = offset_i)
(src/cpu/cpu_backend.cpp:115-147)."""
import numpy as np
import pytest

from gpu_optical_photons_b200 import params as P
from gpu_optical_photons_b200.wavefront import WaveConfig, WavefrontEngine, batched_events
from helpers import check_tally_consistency, chi2_two_sample, compare_histories

pytestmark = pytest.mark.gpu

TC = P.TallyConfig(100, 50.0, 10)


@pytest.fixture(scope="module")
def batch():
    events, counts = batched_events()  # the benchmark's 4096 events
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)
    arr = (P.CSimParams * len(events))(*[e.to_c() for e in events])
    return events, counts, offs, arr


def engine_tallies(events, counts, cfg):
    eng = WavefrontEngine(TC, len(events), int(counts.sum()), cfg)
    try:
        eng.set_events(events, counts)
        eng.run_tally()
        return eng.tallies(), eng.stats()
    finally:
        eng.close()


def test_full_batch_exact_equals_oracle(engine, oracle, batch):
    events, counts, offs, arr = batch
    want = oracle.batch_tally(arr, offs, TC, mode=oracle.PORTABLE)
    assert int(want[:, :5].sum()) == int(counts.sum())
    for cfg in (WaveConfig(math="exact", blocks_per_sm=7, block_size=128),  # the benchmark's variant
                WaveConfig(math="exact")):
        got, st = engine_tallies(events, counts, cfg)
        bad = np.nonzero((got != want).any(axis=1))[0]
        assert len(bad) == 0, f"{len(bad)} events differ, first {bad[:5]} ({cfg})"
        assert st["useful_lane_steps"] == int(want[:, -2].sum() + want[:, -1].sum() + want[:, 1].sum())
    for i in range(0, len(events), 97):
        check_tally_consistency(want[i], TC)
    # The plain history kernel, one launch per event (the benchmark's baseline).
    import torch
    dev = torch.zeros((len(events), TC.length), dtype=torch.int64, device="cuda")
    for i, e in enumerate(events):
        engine.tally_device(e, TC, int(counts[i]), first_id=int(offs[i]), out=dev[i], math="exact")
    hist = dev.cpu().numpy().astype(np.uint64)
    assert np.array_equal(hist, want)


@pytest.fixture(scope="module")
def cpu_platform(oracle, batch):
    events, counts, offs, arr = batch
    return oracle.batch_tally(arr, offs, TC, mode=oracle.PLATFORM)


@pytest.mark.parametrize("math_mode", ["fast", "approx"])
def test_full_batch_fast_agrees_with_cpu(engine, oracle, batch, cpu_platform, math_mode):
    events, counts, offs, arr = batch
    n = int(counts.sum())
    want = cpu_platform
    got, _ = engine_tallies(events, counts, WaveConfig(math=math_mode, blocks_per_sm=7, block_size=128))
    assert int(got[:, :5].sum()) == n
    # Detected photons: |sum over events of the difference| and the sum of
    # per-event |differences|, both within the 0.1 % fate tolerance.
    d_det = got[:, 0].astype(np.int64) - want[:, 0].astype(np.int64)
    assert abs(int(d_det.sum())) <= 1e-3 * n
    assert int(np.abs(d_det).sum()) <= 1e-3 * n
    # Every fate: at least sum|delta| / 2 photons changed fate; bound it.
    d_fate = np.abs(got[:, :5].astype(np.int64) - want[:, :5].astype(np.int64)).sum()
    assert d_fate / 2 <= 1e-3 * n
    t0, x0 = 5, 5 + TC.time_bins + 1
    for lo, hi in ((t0, x0), (x0, x0 + TC.xy_bins ** 2)):
        chi2, ndf, pv = chi2_two_sample(got[:, lo:hi].sum(axis=0), want[:, lo:hi].sum(axis=0))
        assert pv > 0.01, (lo, chi2, ndf)
    # Per-photon fates on a sample of the batch: batched records mode (the same
    # kernel variant) against the oracle's default-math records.
    import torch
    from gpu_optical_photons_b200.backend import device_records, records_to_numpy
    k = 64
    m = int(offs[k])
    eng = WavefrontEngine(TC, k, m, WaveConfig(math=math_mode, blocks_per_sm=7, block_size=128))
    try:
        eng.set_events(events[:k], counts[:k])
        d = device_records(m)
        eng.run_records(d)
        torch.cuda.synchronize()
        rec = records_to_numpy(d)
    finally:
        eng.close()
    ref = {f: [] for f in rec}
    for i in range(k):
        r = oracle.records(events[i], int(counts[i]), int(offs[i]), mode=oracle.PLATFORM)
        for f in ref:
            ref[f].append(r[f])
    ref = {f: np.concatenate(v) for f, v in ref.items()}
    h = compare_histories(rec, ref)
    assert h["fate_differs"] <= 1e-3 * m, h
    assert h["same_discrete"] >= 0.999 * m, h
