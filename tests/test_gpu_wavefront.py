"""Wavefront engine through the C ABI: bit identity with the history kernel (the
property of the reference's tests/test_gpu.cpp:160-212), integer tallies, graph vs
host loop, batched events against the oracle."""
import numpy as np
import pytest

from gpu_optical_photons_b200 import params as P
from gpu_optical_photons_b200.wavefront import WaveConfig, WavefrontEngine, batched_events
from helpers import check_tally_consistency, compare_histories, chi2_two_sample, steps_of

pytestmark = pytest.mark.gpu

SETUPS = {
    "polished": P.SimParams(scat_length=300.0),
    "lambertian": P.SimParams(surface=P.LAMBERTIAN, reflectivity=0.95, n_det=1.5, source=P.VOLUME),
    "capped": P.SimParams(scat_length=300.0, max_steps=5),
}


@pytest.mark.parametrize("setup", list(SETUPS))
@pytest.mark.parametrize("k", [1, 3, 100000])
def test_event_records_identical_to_history(engine, setup, k):
    p = SETUPS[setup]
    n = 100_003
    hist, _ = engine.run_gpu_records(p, n)
    ev, st, _ = engine.run_gpu_records_event(p, n, k, 64, 0, 30011)
    assert compare_histories(hist, ev)["bitwise_identical"] == n
    assert st["useful_lane_steps"] == int(steps_of(hist).sum())
    assert st["issued_lane_steps"] >= st["useful_lane_steps"]


@pytest.mark.parametrize("cfg", [
    WaveConfig(threshold=1), WaveConfig(threshold=32), WaveConfig(threshold=16, cadence=4),
    WaveConfig(threshold=24, wave_quota=50_000), WaveConfig(block_size=128, threshold=8),
    WaveConfig(use_graph=False, threshold=20, cadence=7, wave_quota=30_000)])
@pytest.mark.parametrize("math_mode", ["exact", "fast", "approx"])
def test_wavefront_tally_equals_history_tally(engine, cfg, math_mode):
    p = P.config2()[0]
    c = P.TallyConfig(500, 50.0, 50)
    n = 400_000
    cfg = WaveConfig(**{**cfg.__dict__, "math": math_mode})
    _, fh, _ = engine.run_gpu_tally(p, c, n, math=math_mode)
    eng = WavefrontEngine(c, 1, n, cfg)
    eng.set_events([p], [n])
    eng.run_tally()
    fw = eng.tallies()[0]
    st = eng.stats()
    eng.close()
    assert np.array_equal(fh, fw)
    check_tally_consistency(fw, c)
    assert st["useful_lane_steps"] == int(fh[-2] + fh[-1] + fh[1])


def test_wavefront_records_through_engine(engine):
    import torch
    p = P.config3(True)[0]
    n = 200_000
    hist, _ = engine.run_gpu_records(p, n, first_id=5)
    eng = WavefrontEngine(P.TallyConfig(), 1, n, WaveConfig(threshold=24, cadence=16))
    eng.set_events([p], [n], first_id=5)
    d = engine.device_records(n)
    eng.run_records(d, stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    rec = engine.records_to_numpy(d)
    eng.close()
    assert compare_histories(hist, rec)["bitwise_identical"] == n


def test_batched_events_exact_equals_oracle(engine, oracle):
    events, counts = batched_events(n_events=48, seed=7, median=2000, n_min=1, n_max=20000)
    counts[3] = 0  # an empty event
    counts[10] = 1
    c = P.TallyConfig(100, 50.0, 10)
    eng = WavefrontEngine(c, len(events), int(counts.sum()), WaveConfig(math="exact", threshold=24))
    eng.set_events(events, counts, first_id=1000)
    eng.run_tally()
    got = eng.tallies()
    eng.close()
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64) + np.uint64(1000)
    arr = (P.CSimParams * len(events))(*[e.to_c() for e in events])
    ref = oracle.batch_tally(arr, offs, c, mode=oracle.PORTABLE)
    assert np.array_equal(got, ref)
    for row in got:
        check_tally_consistency(row, c)


@pytest.mark.parametrize("max_steps", [65_535, 65_536, 4_000_000_000])
def test_batched_events_large_step_limits_equal_oracle(engine, oracle, max_steps):
    """Warps cache events in shared-memory slots with 32-bit counters only when
    every event's max_steps is below 2^16 (so one photon adds less than 2^16 to a
    step sum); otherwise every photon adds to its event's 64-bit slice. Both
    paths give the oracle's tallies (exact mode), with a long-lived photon mix
    (mirror-like faces) so step sums are large."""
    events, counts = batched_events(n_events=24, seed=31, median=5000, n_min=1, n_max=40000)
    events = [e.replace(max_steps=max_steps, reflectivity=0.999, abs_length=20000.0) for e in events]
    c = P.TallyConfig(100, 50.0, 10)
    eng = WavefrontEngine(c, len(events), int(counts.sum()), WaveConfig(math="exact"))
    eng.set_events(events, counts, first_id=77)
    eng.run_tally()
    got = eng.tallies()
    eng.close()
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64) + np.uint64(77)
    arr = (P.CSimParams * len(events))(*[e.to_c() for e in events])
    assert np.array_equal(got, oracle.batch_tally(arr, offs, c, mode=oracle.PORTABLE))


def test_batched_events_with_per_face_surfaces(engine, oracle):
    """Events with their own surface model and reflectivity on each face: the
    batched kernel reads a face's reflectivity from the event record by face
    index. Exact mode equals the oracle event by event; fast mode equals the
    history kernel (one configuration per launch, face parameters from the
    kernel argument) event by event."""
    rng = np.random.default_rng(41)
    models = [P.LAMBERTIAN, P.SPECULAR, P.POLISHED, P.BLACK]
    events = []
    for i in range(24):
        fs = [int(models[j]) for j in rng.integers(0, 4, size=5)] + [0]
        fs[i % 5] = P.LAMBERTIAN  # every event keeps at least one painted face
        fr = [float(np.float32(x)) for x in rng.uniform(0.80, 0.99, size=5)] + [0.0]
        events.append(P.SimParams(
            face_surface=fs, face_reflectivity=fr, source=P.VOLUME,
            abs_length=float(np.float32(rng.uniform(300.0, 3000.0))),
            scat_length=float("inf") if i % 2 else float(np.float32(rng.uniform(300.0, 1000.0))),
            n_scint=float(np.float32(rng.uniform(1.5, 1.7)))))
    counts = rng.integers(1, 12_000, size=len(events)).astype(np.uint64)
    counts[7] = 0
    c = P.TallyConfig(100, 50.0, 10)
    first_id = 300
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64) + np.uint64(first_id)
    for math_mode in ("exact", "fast"):
        eng = WavefrontEngine(c, len(events), int(counts.sum()), WaveConfig(math=math_mode))
        eng.set_events(events, counts, first_id=first_id)
        eng.run_tally()
        got = eng.tallies()
        eng.close()
        for i, e in enumerate(events):
            n = int(counts[i])
            if math_mode == "exact":
                want = oracle.tally(e, c, n, int(offs[i]), mode=oracle.PORTABLE)
            else:
                want = engine.tally_device(e, c, n, first_id=int(offs[i]), math="fast").cpu().numpy()
            assert np.array_equal(got[i], want.astype(np.uint64)), (math_mode, i, e.face_surface)
            assert int(got[i, :5].sum()) == n


def test_batched_records_exact_bitwise_equal_oracle(engine, oracle):
    """Per-photon records of a batch (the batched records variant of the wave
    kernel, each photon reading its event's record) equal the oracle's records of
    each event bit for bit in exact mode, in batch order."""
    import torch
    events, counts = batched_events(n_events=16, seed=43, median=3000, n_min=1, n_max=15000)
    events[5] = events[5].replace(face_surface=[P.SPECULAR, P.BLACK, P.LAMBERTIAN, P.POLISHED, P.LAMBERTIAN, 0],
                                  face_reflectivity=[0.97, 0.5, 0.9, 0.8, 0.93, 0.0],
                                  scat_length=450.0, source=P.VOLUME)
    counts[9] = 0
    n = int(counts.sum())
    first_id = 4242
    eng = WavefrontEngine(P.TallyConfig(100, 50.0, 10), len(events), n, WaveConfig(math="exact"))
    try:
        eng.set_events(events, counts, first_id=first_id)
        d = engine.device_records(n)
        eng.run_records(d)
        torch.cuda.synchronize()
        rec = engine.records_to_numpy(d)
    finally:
        eng.close()
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    for i, e in enumerate(events):
        lo, hi = int(offs[i]), int(offs[i + 1])
        if hi == lo:
            continue
        want = oracle.records(e, hi - lo, first_id + lo, mode=oracle.PORTABLE)
        got = {k: rec[k][lo:hi] for k in rec}
        h = compare_histories(got, want)
        assert h["bitwise_identical"] == hi - lo, (i, h)


@pytest.mark.parametrize("math_mode", ["exact", "fast"])
def test_batched_shared_physics_equals_oracle(engine, oracle, math_mode):
    """Events with the same step physics but their own sources, decay times and
    photon counts run the shared-physics batched variant; the per-event tallies
    equal the oracle's (exact mode) or agree in detection (fast mode)."""
    rng = np.random.default_rng(23)
    base = P.SimParams(surface=P.LAMBERTIAN, reflectivity=0.93, n_det=1.5, scat_length=400.0,
                       abs_length=1500.0)
    events = [base.replace(src_x=float(rng.uniform(-20, 20)), src_y=float(rng.uniform(-20, 20)),
                           src_z=float(rng.uniform(-20, 20)), tau=float(rng.uniform(1, 6)),
                           source=P.VOLUME if i % 5 == 0 else P.POINT) for i in range(30)]
    counts = rng.integers(0, 20_000, len(events))
    c = P.TallyConfig(100, 50.0, 10)
    eng = WavefrontEngine(c, len(events), int(counts.sum()), WaveConfig(math=math_mode))
    eng.set_events(events, counts, first_id=321)
    eng.run_tally()
    got = eng.tallies()
    eng.close()
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64) + np.uint64(321)
    arr = (P.CSimParams * len(events))(*[e.to_c() for e in events])
    ref = oracle.batch_tally(arr, offs, c, mode=oracle.PORTABLE if math_mode == "exact" else oracle.PLATFORM)
    assert np.array_equal(got[:, :5].sum(1), counts)
    if math_mode == "exact":
        assert np.array_equal(got, ref)
    else:
        assert np.abs(got[:, 0].astype(np.int64) - ref[:, 0].astype(np.int64)).sum() <= 0.001 * counts.sum()


@pytest.mark.parametrize("chunk", [32, 33, 1000, 65536])
@pytest.mark.parametrize("bins", [(100, 10), (300, 12)])  # bins cached per warp / global bins
def test_batched_tallies_independent_of_chunk(engine, oracle, chunk, bins):
    events, counts = batched_events(n_events=40, seed=19, median=3000, n_min=1, n_max=30000)
    counts[5] = 0
    c = P.TallyConfig(bins[0], 50.0, bins[1])
    eng = WavefrontEngine(c, len(events), int(counts.sum()),
                          WaveConfig(math="exact", threshold=26, chunk=chunk))
    eng.set_events(events, counts)
    eng.run_tally()
    got = eng.tallies()
    eng.close()
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)
    arr = (P.CSimParams * len(events))(*[e.to_c() for e in events])
    assert np.array_equal(got, oracle.batch_tally(arr, offs, c, mode=oracle.PORTABLE))


def test_chunk_out_of_range_rejected(engine):
    from gpu_optical_photons_b200._lib import InvalidArgument
    for chunk in (16, (1 << 20) + 1):
        with pytest.raises(InvalidArgument):
            WavefrontEngine(P.TallyConfig(), 1, 100, WaveConfig(chunk=chunk))


def test_batched_events_fast_vs_oracle(engine, oracle):
    events, counts = batched_events(n_events=64, seed=11, median=5000)
    c = P.TallyConfig(100, 50.0, 10)
    eng = WavefrontEngine(c, len(events), int(counts.sum()))
    got, st, tm = eng.run_batch(events, counts)
    eng.close()
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)
    arr = (P.CSimParams * len(events))(*[e.to_c() for e in events])
    ref = oracle.batch_tally(arr, offs, c, mode=oracle.PLATFORM)
    assert np.array_equal(got[:, :5].sum(1), counts)
    # per-event detected counts agree to the floating-point divergence tolerance
    assert np.abs(got[:, 0].astype(np.int64) - ref[:, 0].astype(np.int64)).sum() <= 0.001 * counts.sum()
    chi2, ndf, pv = chi2_two_sample(got[:, 5:106].sum(0), ref[:, 5:106].sum(0))
    assert pv > 0.01


def test_graph_and_host_loop_agree(engine):
    events, counts = batched_events(n_events=32, seed=3, median=3000)
    c = P.TallyConfig(100, 50.0, 10)
    out = []
    for g in (True, False):
        eng = WavefrontEngine(c, 32, int(counts.sum()), WaveConfig(use_graph=g, wave_quota=20000))
        eng.set_events(events, counts)
        eng.run_tally()
        out.append(eng.tallies())
        eng.close()
    assert np.array_equal(out[0], out[1])


def test_run_batch_with_event_table(engine):
    """A batch converted once (EventTable) gives the same tallies as the list."""
    from gpu_optical_photons_b200.wavefront import EventTable
    events, counts = batched_events(n_events=48, median=2e3)
    tc = P.TallyConfig(100, 50.0, 10)
    eng = WavefrontEngine(tc, len(events), int(counts.sum()))
    try:
        a, _, _ = eng.run_batch(events, counts)
        tab = EventTable(events)
        b, _, _ = eng.run_batch(tab, counts)
        eng.set_events(tab, counts)
        eng.run_tally()
        c = eng.tallies()
    finally:
        eng.close()
    assert np.array_equal(a, b) and np.array_equal(a, c)


def test_tally_just_under_the_default_shared_memory_limit(engine, oracle):
    """A tally whose histograms bring the wave kernel's dynamic shared memory to
    49,072 B: below 48 KB, but above 48 KB minus the kernel's static shared memory,
    so the launch needs the opt-in attribute all the same."""
    p = P.config2()[0]
    c = P.TallyConfig(5098, 50.0, 1)  # 5 + 5099 + 1 + 2 entries; bins 5100 x 4 B + 8 pantries x 3584 B
    n = 100_000
    want = oracle.tally(p, c, n, 9, mode=oracle.PORTABLE)
    eng = WavefrontEngine(c, 1, n, WaveConfig(math="exact"))
    try:
        eng.set_events([p], [n], first_id=9)
        eng.run_tally()
        assert np.array_equal(eng.tallies()[0], want)
    finally:
        eng.close()
    _, flat, _ = engine.run_gpu_tally(p, c, n, first_id=9, math="exact")
    assert np.array_equal(flat, want)


def test_tally_at_the_top_of_shared_memory(engine, oracle):
    """Histograms that fit the opt-in shared memory per block beside the pantries
    of 8 warps only if the kernel's static shared memory is forgotten: the engine
    refuses them with a clear error (no CUDA error), and the host tally call still
    answers, bit for bit (history kernel or the 4-warp engine of the host calls)."""
    import torch
    props = torch.cuda.get_device_properties(0)
    optin = int(getattr(props, "shared_memory_per_block_optin", 232448))
    n_bins = (optin - 8 * 3584) // 4 - 6  # dynamic bytes within the kernel's static size of the limit
    c = P.TallyConfig(n_bins - 2, 50.0, 1)  # time bins + overflow + 1 hit-map bin = n_bins
    with pytest.raises(engine.OptxError, match="shared memory"):
        WavefrontEngine(c, 1, 1000, WaveConfig(math="exact"))
    p = P.config1()[0]
    _, flat, _ = engine.run_gpu_tally(p, c, 20_000, first_id=3, math="exact")
    assert np.array_equal(flat, oracle.tally(p, c, 20_000, 3, mode=oracle.PORTABLE))
