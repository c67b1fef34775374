"""Genstep emission in the oracle (CPU).

Gensteps are an extension (the reference has no counterpart; its README lists
generation from gensteps as future work), so their bitwise parity is with the
oracle's restatement of the package's own definition (the GPU tests). Here the
oracle is checked against the reference statistically: a degenerate genstep (a
zero-length segment at (sx, sy, sz), t0 = t1 = 0) emits the photons of the
reference's point source at (sx, sy, sz) — same place, isotropic directions, the
same decay time law — from other words of the Philox stream (a genstep draws six
emission words, the point source three), so fates, arrival times and hit map
must agree in distribution with the reference CPU build's point-source run.
"""
import numpy as np
import pytest

from gpu_optical_photons_b200 import compare as C
from gpu_optical_photons_b200 import gensteps as G
from gpu_optical_photons_b200 import params as P


def _point_gensteps(sources, counts, event_of):
    g = np.zeros(len(counts), G.GENSTEP_DTYPE)
    for i, ((x, y, z), n, e) in enumerate(zip(sources, counts, event_of)):
        g[i] = (x, y, z, 0.0, x, y, z, 0.0, n, e)
    return g


def test_degenerate_gensteps_match_reference_point_source(oracle):
    if not oracle.ref_available(oracle.PLATFORM):
        pytest.skip("reference CPU build (oracle/_ref) not present")
    ev = P.SimParams(surface=P.LAMBERTIAN, reflectivity=0.95, n_det=1.5, scat_length=500.0, tau=4.0,
                     src_x=10.0, src_y=-5.0, src_z=3.0)
    n = 200_000
    g = _point_gensteps([(10.0, -5.0, 3.0)] * 4, [n // 4] * 4, [0] * 4)
    _, rg = oracle.genstep_run([ev], g, None, first_id=0, records=True, mode=oracle.PLATFORM)
    rr = oracle.ref_records(ev, n, 0, mode=oracle.PLATFORM)[0]
    assert np.all(rg["fate"] <= 4)
    d = C.compare_distributions(rr, rg, ev, time_bins=100, t_max=50.0, xy_bins=10)
    assert abs(d.eff_z) < 4.0
    assert d.time_chi2.pvalue > 1e-4 and d.xy_chi2.pvalue > 1e-4 and d.time_ks.pvalue > 1e-4
    for f in range(5):  # every fate fraction within 4 sigma
        a, b = np.mean(rr["fate"] == f), np.mean(rg["fate"] == f)
        s = np.sqrt((a * (1 - a) + b * (1 - b)) / n) + 1e-12
        assert abs(a - b) < 4 * s + 1e-9, f


def test_genstep_records_lie_on_their_segments(oracle):
    ev = [P.SimParams(abs_length=1e-6)]  # absorbed at once: the record is the emission point
    g = np.zeros(2, G.GENSTEP_DTYPE)
    g[0] = (-10, 0, 5, 1.0, 10, 4, 5, 3.0, 4000, 0)
    g[1] = (0, -20, -20, 7.0, 0, 20, 20, 7.0, 4000, 0)
    _, r = oracle.genstep_run(ev, g, None, records=True, mode=oracle.PORTABLE)
    a = slice(0, 4000)
    assert np.all(r["fate"] == P.ABSORBED_BULK)
    f = (r["x"][a] + 10) / 20
    assert np.allclose(r["y"][a], 4 * f, atol=1e-3) and np.allclose(r["z"][a], 5.0)
    assert 0.0 <= f.min() and f.max() <= 1.0 and f.std() > 0.25  # uniform on [0, 1]
    assert r["t"][a].min() >= 1.0  # window start + decay
    b = slice(4000, 8000)
    assert np.allclose(r["x"][b], 0.0, atol=1e-4) and np.allclose(r["y"][b], r["z"][b], atol=1e-3)
    assert r["t"][b].min() >= 7.0


def test_gensteps_route_to_their_events(oracle):
    events, g = G.muon_events(6, seed=3, photons_per_mm=40.0, step_mm=5.0)
    c = P.TallyConfig(50, 50.0, 5)
    t, _ = oracle.genstep_run(events, g, c, mode=oracle.PORTABLE)
    per_event = np.bincount(g["event"], weights=g["n_photons"], minlength=6)
    assert np.array_equal(t[:, :5].sum(1), per_event.astype(np.uint64))
    # shuffling the genstep order moves photon ids but keeps each event's photon count
    perm = np.random.default_rng(0).permutation(len(g))
    t2, _ = oracle.genstep_run(events, g[perm], c, mode=oracle.PORTABLE)
    assert np.array_equal(t2[:, :5].sum(1), t[:, :5].sum(1))


def test_track_gensteps_shape():
    g = G.track_gensteps((0, 0, -25), (0, 0, 25), photons_per_mm=100.0, step_mm=2.0,
                         rng=np.random.default_rng(1))
    assert len(g) == 25
    assert np.allclose(g["z1"] - g["z0"], 2.0)
    assert np.all(g["t1"] > g["t0"])
    assert abs(g["n_photons"].mean() - 200) < 20
    assert G.as_gensteps(list(map(tuple, g.tolist()))).tobytes() == g.tobytes()
