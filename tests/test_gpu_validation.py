"""Analytic validation on the GPU: the reference's tests/test_transport_cpu.cpp
cases V1-V5b (solid angle per face, hit map, time of flight, absorption,
Rayleigh, volume source, escape cone, lossless diffuse box), run through the
history kernel and the wavefront engine. Thresholds as in the reference:
|pull| < 4, p > 1e-4."""
import math

import numpy as np
import pytest
from scipy import stats as ss

from gpu_optical_photons_b200 import params as P
from gpu_optical_photons_b200.wavefront import WaveConfig, wavefront_tally
from helpers import (binomial_pull, face_solid_angle_fraction, face_survival_fraction,
                     mirror_box_escape_fraction, rect_solid_angle)

pytestmark = pytest.mark.gpu


def face_of(r, p):
    f = np.full(len(r["x"]), -1)
    for face, (arr, val) in enumerate([(r["x"], -p.hx), (r["x"], p.hx), (r["y"], -p.hy),
                                       (r["y"], p.hy), (r["z"], -p.hz), (r["z"], p.hz)]):
        f[(f < 0) & (arr == np.float32(val))] = face
    return f


@pytest.mark.parametrize("case", [(0, 0, 0, 50, 50, 50), (10, -5, 3, 50, 50, 50), (0, 0, 20, 50, 50, 50),
                                  (20, 20, -20, 50, 50, 50), (5, 10, -4, 30, 50, 20)])
def test_v1_solid_angle_every_face(engine, case):
    sx, sy, sz, X, Y, Z = case
    p = P.black_box().replace(src_x=sx, src_y=sy, src_z=sz, hx=X / 2, hy=Y / 2, hz=Z / 2,
                              seed=1000 + int(sx * 7 + sy * 3 + sz))
    n = 2_000_000
    rec, _ = engine.run_gpu_records(p, n)
    f = face_of(rec, p)
    assert (f >= 0).all()
    assert (rec["n_boundary"] == 1).all() and (rec["n_scatter"] == 0).all()
    assert np.array_equal(rec["fate"] == P.DETECTED, f == 5)
    for face in range(6):
        pull = binomial_pull(int((f == face).sum()), n, face_solid_angle_fraction(p, face))
        assert abs(pull) < 4, (face, pull)


def test_v1b_hit_map_chi2(engine):
    p = P.black_box().replace(src_x=5.0, src_y=-3.0, src_z=-10.0, seed=2024)
    n = 4_000_000
    rec, _ = engine.run_gpu_records(p, n)
    d = rec["fate"] == P.DETECTED
    kb = 20
    obs = np.histogram2d(rec["y"][d], rec["x"][d], bins=kb, range=[[-p.hy, p.hy], [-p.hx, p.hx]])[0]
    exp = np.zeros((kb, kb))
    h = p.hz - p.src_z
    for iy in range(kb):
        for ix in range(kb):
            x1 = -p.hx + 2 * p.hx * ix / kb - p.src_x
            y1 = -p.hy + 2 * p.hy * iy / kb - p.src_y
            exp[iy, ix] = n * rect_solid_angle(x1, x1 + 2 * p.hx / kb, y1, y1 + 2 * p.hy / kb, h) / (4 * math.pi)
    chi2 = float(((obs - exp) ** 2 / exp).sum())
    assert ss.chi2.sf(chi2, kb * kb) > 1e-4


def test_v1c_time_of_flight(engine):
    p = P.black_box().replace(src_x=-7.0, src_y=4.0, src_z=2.0, tau=4.0, seed=77)
    n = 500_000
    rec, _ = engine.run_gpu_records(p, n)
    r = np.sqrt((rec["x"] - p.src_x) ** 2 + (rec["y"] - p.src_y) ** 2 + (rec["z"] - p.src_z) ** 2)
    assert np.allclose(rec["path"], r, rtol=1e-5)
    t_emit = rec["t"] - rec["path"].astype(np.float64) * (np.float32(p.n_scint) / 299.792458)
    assert ss.kstest(t_emit, lambda t: 1 - np.exp(-t / p.tau)).pvalue > 1e-4


@pytest.mark.parametrize("L", [20.0, 100.0, 1000.0])
@pytest.mark.parametrize("engine_kind", ["history", "wave"])
def test_v2_absorption(engine, L, engine_kind):
    p = P.black_box().replace(abs_length=L, src_x=6.0, src_y=-8.0, src_z=-5.0, seed=500 + int(L))
    n = 2_000_000
    c = P.TallyConfig()
    if engine_kind == "history":
        t, _, _ = engine.run_gpu_tally(p, c, n)
    else:
        t, _, _ = wavefront_tally(p, c, n)
    p_det = face_survival_fraction(p, 5, L)
    p_abs = 1 - sum(face_survival_fraction(p, f, L) for f in range(6))
    assert abs(binomial_pull(int(t.fate_counts[0]), n, p_det)) < 4
    assert abs(binomial_pull(int(t.fate_counts[1]), n, p_abs)) < 4


@pytest.mark.parametrize("engine_kind", ["history", "wave"])
def test_v3_rayleigh_symmetric_cube(engine, engine_kind):
    p = P.black_box().replace(scat_length=15.0, seed=31)
    n = 2_000_000
    rec, _ = engine.run_gpu_records(p, n)
    c = np.bincount(rec["fate"], minlength=5)
    assert c[0] + c[2] == n
    assert abs(binomial_pull(int(c[0]), n, 1 / 6)) < 4
    unscattered = int(((rec["fate"] == 0) & (rec["n_scatter"] == 0)).sum())
    assert abs(binomial_pull(unscattered, n, face_survival_fraction(p, 5, 15.0))) < 4
    assert int(rec["n_scatter"].sum()) > n
    if engine_kind == "wave":
        t, _, st = wavefront_tally(p, P.TallyConfig(), n)
        assert np.array_equal(t.fate_counts, c) and t.scatter_sum == int(rec["n_scatter"].sum())


def test_v4_volume_source(engine):
    p = P.black_box().replace(source=P.VOLUME, seed=4)
    n = 2_000_000
    t, _, _ = engine.run_gpu_tally(p, P.TallyConfig(), n)
    assert abs(binomial_pull(int(t.fate_counts[0]), n, 1 / 6)) < 4


@pytest.mark.parametrize("engine_kind", ["history", "wave"])
def test_v5_mirror_box_escape_cone(engine, engine_kind):
    p = P.SimParams(surface=P.SPECULAR, reflectivity=1.0, n_det=1.0, abs_length=P.INF,
                    scat_length=P.INF, max_steps=1000, src_x=3.0, src_y=-11.0, src_z=7.0, seed=5)
    n = 200_000
    if engine_kind == "history":
        t, _, _ = engine.run_gpu_tally(p, P.TallyConfig(), n)
    else:
        t, _, _ = wavefront_tally(p, P.TallyConfig(), n, config=WaveConfig(threshold=16))
    c = t.fate_counts
    assert abs(binomial_pull(int(c[0]), n, mirror_box_escape_fraction(p.n_scint, p.n_det))) < 4
    assert c[0] + c[4] == n  # detected or trapped (max_steps), nothing else


def test_v5b_lossless_lambertian_detects_all(engine):
    p = P.SimParams(surface=P.LAMBERTIAN, reflectivity=1.0, n_det=1.0, abs_length=P.INF, seed=6)
    n = 200_000
    t, _, _ = wavefront_tally(p, P.TallyConfig(), n)
    assert int(t.fate_counts[0]) == n


def test_per_face_black_bar_against_oracle_fractions(engine, oracle):
    """Config 3 (-z black): the wavefront tally agrees with the oracle statistically."""
    p, c = P.config3(True)
    n = 2_000_000
    t, flat, _ = wavefront_tally(p, c, n)
    ref = oracle.tally(p.replace(seed=p.seed + 1), c, n)
    for f in range(4):
        a, b = int(flat[f]), int(ref[f])
        if a + b == 0:
            continue
        pa, pb = a / n, b / n
        z = (pa - pb) / math.sqrt(max(pa * (1 - pa) / n + pb * (1 - pb) / n, 1e-300))
        assert abs(z) < 4, (f, z)
