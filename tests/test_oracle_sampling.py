"""The transport's direction samplers on the oracle (the reference's sampling
cases, tests/test_sampling.cpp: isotropic, Lambertian, Rayleigh; CPU):
unit length, and the distributions of the polar cosine and the azimuth."""
import ctypes

import numpy as np
from scipy import stats

N = 40_000


def _draw(oracle, kind, axis):
    f = oracle.lib().oracle_sample_direction
    rng = np.random.default_rng(1234 + kind)
    u = ((rng.integers(0, 1 << 24, size=(N, 2)) + 1) * 2.0 ** -24).astype(np.float32)  # (0, 1]
    a = (ctypes.c_float * 3)(*axis)
    out = (ctypes.c_float * 3)()
    d = np.empty((N, 3))
    for i in range(N):
        f(kind, float(u[i, 0]), float(u[i, 1]), a, out)
        d[i] = out[:]
    return d


def _uniform_p(x):
    """Chi-squared p-value of x against uniform on [0, 1] in 50 bins."""
    h = np.bincount(np.minimum((x * 50).astype(int), 49), minlength=50)
    return stats.chisquare(h).pvalue


AXIS = np.array([0.3, -0.5, 0.8]) / np.linalg.norm([0.3, -0.5, 0.8])


def test_isotropic(oracle):
    d = _draw(oracle, 0, (0.0, 0.0, 1.0))
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-6)
    assert _uniform_p((d[:, 2] + 1.0) / 2.0) > 1e-4                        # cos theta uniform
    assert _uniform_p((np.arctan2(d[:, 1], d[:, 0]) + np.pi) / (2 * np.pi)) > 1e-4   # azimuth uniform


def test_lambertian_is_cosine_weighted(oracle):
    d = _draw(oracle, 1, tuple(np.float32(AXIS)))
    mu = d @ AXIS
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-5)
    assert mu.min() >= -1e-6                                                # the hemisphere of the axis
    assert _uniform_p(np.clip(mu, 0.0, 1.0) ** 2) > 1e-4                    # P(mu) = 2 mu: mu^2 uniform


def test_rayleigh_phase_function(oracle):
    d = _draw(oracle, 2, tuple(np.float32(AXIS)))
    mu = np.clip(d @ AXIS, -1.0, 1.0)
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-5)
    # 3/8 (1 + mu^2): CDF (mu^3 + 3 mu + 4) / 8 is uniform; <mu> = 0, <mu^2> = 2/5,
    # var(mu^2) = <mu^4> - <mu^2>^2 = 9/35 - 4/25
    assert _uniform_p((mu ** 3 + 3 * mu + 4) / 8) > 1e-4
    assert abs(mu.mean()) < 5 * np.sqrt(2 / 5 / N)
    assert abs((mu ** 2).mean() - 0.4) < 5 * np.sqrt((9 / 35 - 4 / 25) / N)
