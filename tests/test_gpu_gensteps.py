"""Gensteps on the GPU (optx_engine_set_gensteps / optx_run_gensteps).

Exact mode equals the oracle's genstep restatement bit for bit (per-event
tallies and per-photon records, in photon order); fast mode agrees with it in
fates (>= 99.9 % per photon) and in distribution; tallies do not depend on the
genstep order within the engine's scheduling knobs (chunk, threshold, graph or
host loop), only on the photon ids, which follow the genstep order.
"""
import numpy as np
import pytest

from gpu_optical_photons_b200 import gensteps as G
from gpu_optical_photons_b200 import params as P
from gpu_optical_photons_b200._lib import InvalidArgument
from gpu_optical_photons_b200.wavefront import WaveConfig, WavefrontEngine
from helpers import check_tally_consistency, compare_histories

pytestmark = pytest.mark.gpu

TC = P.TallyConfig(100, 50.0, 10)


def _workload(n_events=24, seed=5, ppm=60.0, step=2.5):
    events, g = G.muon_events(n_events, seed=seed, photons_per_mm=ppm, step_mm=step)
    g["n_photons"][::17] = 0  # some empty gensteps
    perm = np.random.default_rng(seed).permutation(len(g))  # events interleaved
    return events, g[perm]


def _engine(events, g, max_photons=0, **cfg):
    kw = {"math": "exact", "max_gensteps": len(g), **cfg}
    return WavefrontEngine(TC, len(events), max(G.photons_of(g), max_photons, 1), WaveConfig(**kw))


@pytest.mark.parametrize("cfg", [{}, {"chunk": 32, "threshold": 32}, {"chunk": 4096, "threshold": 8},
                                 {"use_graph": False, "cadence": 3}])
def test_genstep_tallies_exact_equal_oracle(engine, oracle, cfg):
    events, g = _workload()
    eng = _engine(events, g, **cfg)
    eng.set_gensteps(events, g, first_id=123)
    eng.run_tally()
    got = eng.tallies()
    eng.close()
    ref, _ = oracle.genstep_run(events, g, TC, first_id=123, mode=oracle.PORTABLE)
    assert got.shape == (len(events), TC.length)
    assert np.array_equal(got, ref)
    for row in got:
        check_tally_consistency(row, TC)


def test_genstep_events_with_per_face_surfaces_exact_equal_oracle(engine, oracle):
    """Gensteps emitting into events whose faces have their own surface model and
    reflectivity (each photon reads its face parameters from its event's record)."""
    events, g = _workload(n_events=12, seed=23)
    rng = np.random.default_rng(23)
    models = [P.LAMBERTIAN, P.SPECULAR, P.POLISHED, P.BLACK]
    events = [e.replace(face_surface=[int(models[j]) for j in rng.integers(0, 4, size=5)] + [0],
                        face_reflectivity=[float(np.float32(x)) for x in rng.uniform(0.8, 0.99, 5)] + [0.0])
              for e in events]
    eng = _engine(events, g)
    eng.set_gensteps(events, g, first_id=61)
    eng.run_tally()
    got = eng.tallies()
    eng.close()
    ref, _ = oracle.genstep_run(events, g, TC, first_id=61, mode=oracle.PORTABLE)
    assert np.array_equal(got, ref)


def test_genstep_records_exact_equal_oracle(engine, oracle):
    import torch
    events, g = _workload(n_events=8, ppm=30.0)
    n = G.photons_of(g)
    eng = _engine(events, g, threshold=24)
    eng.set_gensteps(events, g, first_id=9)
    d = engine.device_records(n)
    eng.run_records(d, stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    rec = engine.records_to_numpy(d)
    eng.close()
    _, ref = oracle.genstep_run(events, g, None, first_id=9, mode=oracle.PORTABLE, records=True)
    assert compare_histories(ref, rec)["bitwise_identical"] == n


def test_small_gensteps_fine_event_table(engine, oracle):
    """Gensteps of 1..5 photons: the photon -> genstep table runs at its finest
    resolution and every photon still finds its genstep."""
    rng = np.random.default_rng(2)
    events = [P.SimParams(surface=P.LAMBERTIAN, n_det=1.5, scat_length=300.0)] * 3
    g = np.zeros(20_000, G.GENSTEP_DTYPE)
    g["x0"], g["y0"], g["z0"] = rng.uniform(-20, 20, (3, len(g)))
    g["x1"], g["y1"], g["z1"] = g["x0"] + 1, g["y0"], g["z0"] - 1
    g["t1"] = 2.0
    g["n_photons"] = rng.integers(1, 6, len(g))
    g["event"] = rng.integers(0, 3, len(g))
    eng = _engine(events, g)
    out, st, tm = eng.run_gensteps(events, g)
    eng.close()
    ref, _ = oracle.genstep_run(events, g, TC, mode=oracle.PORTABLE)
    assert np.array_equal(out, ref)
    assert st["useful_lane_steps"] > 0


def test_single_genstep_and_fast_mode(engine, oracle):
    events = [P.config2()[0]]
    g = np.zeros(1, G.GENSTEP_DTYPE)
    g[0] = (-20, 0, 0, 0, 20, 0, 0, 5.0, 200_000, 0)
    eng = _engine(events, g, math="fast")
    eng.set_gensteps(events, g)
    eng.run_tally()
    got = eng.tallies()
    eng.close()
    ref, _ = oracle.genstep_run(events, g, TC, mode=oracle.PLATFORM)
    assert got[0, :5].sum() == 200_000
    assert abs(int(got[0, 0]) - int(ref[0, 0])) <= 0.001 * 200_000


def test_fast_mode_records_agree_with_oracle(engine, oracle):
    import torch
    events, g = _workload(n_events=6, ppm=40.0)
    n = G.photons_of(g)
    eng = _engine(events, g, math="fast")
    eng.set_gensteps(events, g)
    d = engine.device_records(n)
    eng.run_records(d, stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    rec = engine.records_to_numpy(d)
    eng.close()
    _, ref = oracle.genstep_run(events, g, None, mode=oracle.PLATFORM, records=True)
    h = compare_histories(ref, rec)
    assert h["fate_differs"] <= 0.001 * n


def test_genstep_errors(engine):
    events, g = _workload(n_events=2)
    eng = _engine(events, g)
    bad = g.copy()
    bad["event"][0] = 5
    with pytest.raises(InvalidArgument):
        eng.set_gensteps(events, bad)
    bad = g.copy()
    bad["t1"][1] = bad["t0"][1] - 1.0
    with pytest.raises(InvalidArgument):
        eng.set_gensteps(events, bad)
    bad = g.copy()
    bad["x0"][2] = np.nan
    with pytest.raises(InvalidArgument):
        eng.set_gensteps(events, bad)
    with pytest.raises(InvalidArgument):
        eng.set_gensteps(events, np.concatenate([g, g]))  # more than max_gensteps
    eng.close()
    eng = WavefrontEngine(TC, 2, 1000)  # no genstep capacity
    with pytest.raises(InvalidArgument):
        eng.set_gensteps(events, g[:1])
    eng.close()


def test_set_events_after_gensteps(engine, oracle):
    """The same engine runs gensteps, then plain events, then gensteps again."""
    events, g = _workload(n_events=4, ppm=20.0)
    eng = _engine(events, g, max_photons=10_000)
    eng.set_gensteps(events, g)
    eng.run_tally()
    a = eng.tallies()
    counts = [1000, 0, 2500, 10]
    evs = [P.SimParams(n_det=1.5), P.SimParams(), P.config2()[0], P.SimParams(surface=P.BLACK)]
    eng.set_events(evs, counts)
    eng.run_tally()
    b = eng.tallies()
    eng.set_gensteps(events, g)
    eng.run_tally()
    c = eng.tallies()
    eng.close()
    assert np.array_equal(a, c)
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)
    arr = (P.CSimParams * 4)(*[e.to_c() for e in evs])
    assert np.array_equal(b, oracle.batch_tally(arr, offs, TC, mode=oracle.PORTABLE))


@pytest.mark.parametrize("cfg", [{}, {"use_graph": False, "cadence": 3}, {"math": "fast"}])
def test_device_gensteps_equal_host_gensteps(engine, oracle, cfg):
    """Gensteps uploaded from device memory give the host upload's tallies and
    records, bit for bit (exact mode: the oracle's too)."""
    import torch
    events, g = _workload()
    n = G.photons_of(g)
    eng = _engine(events, g, **cfg)
    try:
        eng.set_gensteps(events, g, first_id=77)
        eng.run_tally()
        host = eng.tallies()
        dh = engine.device_records(n)
        eng.run_records(dh)
        dg = G.to_device(g)
        stream = torch.cuda.current_stream().cuda_stream
        eng.set_gensteps_device(events, dg, first_id=77, stream=stream)
        eng.run_tally(stream=stream)
        dev = eng.tallies(stream=stream)
        dd = engine.device_records(n)
        eng.run_records(dd, stream=stream)
        torch.cuda.synchronize()
    finally:
        eng.close()
    assert np.array_equal(dev, host)
    rh, rd = engine.records_to_numpy(dh), engine.records_to_numpy(dd)
    assert compare_histories(rd, rh)["bitwise_identical"] == n
    if cfg.get("math", "exact") == "exact":
        ref, _ = oracle.genstep_run(events, g, TC, first_id=77, mode=oracle.PORTABLE)
        assert np.array_equal(dev, ref)


def test_device_gensteps_many_tiles(engine):
    """More gensteps than one scan tile (4096): the two-level photon-offset scan."""
    events, g = G.muon_events(64, seed=9, photons_per_mm=4.0, step_mm=0.25)
    assert len(g) > 2 * 4096  # three tiles
    eng = _engine(events, g, math="fast")
    try:
        eng.set_gensteps(events, g)
        eng.run_tally()
        host = eng.tallies()
        eng.set_gensteps_device(events, G.to_device(g))
        eng.run_tally()
        assert np.array_equal(eng.tallies(), host)
    finally:
        eng.close()


def test_device_genstep_errors_reported_on_the_device(engine):
    """An invalid device genstep, or more photons than the engine holds, is
    reported by the next tallies(); a valid upload afterwards runs normally."""
    events, g = _workload(n_events=6)
    eng = _engine(events, g)
    try:
        eng.set_gensteps(events, g)
        eng.run_tally()
        good = eng.tallies()
        for bad_field, value in (("event", len(events)), ("t1", -1.0), ("x0", np.nan)):
            b = g.copy()
            b[bad_field][3] = value
            eng.set_gensteps_device(events, G.to_device(b))
            eng.run_tally()
            with pytest.raises(InvalidArgument):
                eng.tallies()
        big = g.copy()
        big["n_photons"][0] = eng.max_photons  # over the engine's capacity
        eng.set_gensteps_device(events, G.to_device(big))
        eng.run_tally()
        with pytest.raises(InvalidArgument):
            eng.tallies()
        with pytest.raises(InvalidArgument):  # more than max_gensteps: rejected on the host
            _lib_call_too_many(eng, events)
        eng.set_gensteps_device(events, G.to_device(g))
        eng.run_tally()
        assert np.array_equal(eng.tallies(), good)
    finally:
        eng.close()


def _lib_call_too_many(eng, events):
    import ctypes
    import torch
    from gpu_optical_photons_b200 import _lib
    from gpu_optical_photons_b200.wavefront import _events_c
    arr, faces = _events_c(events)
    dummy = torch.zeros(40, dtype=torch.uint8, device="cuda")
    _lib.call("optx_engine_set_gensteps_device", eng._h, ctypes.cast(arr, ctypes.c_void_p), None,
              len(events), ctypes.c_void_p(dummy.data_ptr()), eng.config.max_gensteps + 1, 0, None)


def test_genstep_ranges_equal_one_run(engine, oracle):
    """A genstep batch run as photon ranges (checkpoint and resume) gives the
    one-run tallies; ranges are refused after a device-genstep upload, whose
    photon total the host does not know."""
    events, g = _workload(seed=9)
    n = G.photons_of(g)
    eng = _engine(events, g)
    try:
        eng.set_gensteps(events, g, first_id=55)
        for i, (lo, hi) in enumerate([(0, n // 5), (n // 5, n // 2), (n // 2, n)]):
            eng.run_tally_range(lo, hi, accumulate=i > 0)
        got = eng.tallies()
        ref, _ = oracle.genstep_run(events, g, TC, first_id=55, mode=oracle.PORTABLE)
        assert np.array_equal(got, ref)
        eng.set_gensteps_device(events, G.to_device(g), first_id=55)
        with pytest.raises(InvalidArgument, match="photon ranges"):
            eng.run_tally_range(0, 10)
    finally:
        eng.close()
