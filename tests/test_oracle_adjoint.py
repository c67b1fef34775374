"""The oracle's FP64 score-function terms, on the CPU: the per-bin score
moments agree with the weighted gradient sum, the decay-time score averages to
zero over detected photons (the emission time does not change detection), and
the absorption-length score matches common-random-number finite differences of
the detected fraction."""
import math

import numpy as np

from gpu_optical_photons_b200 import params as P

TC = P.TallyConfig(500, 50.0, 1)


def test_score_moments_match_the_weighted_gradient(oracle):
    p = P.config2()[0].replace(abs_length=1000.0, scat_length=700.0, tau=4.0)
    n = 40_000
    w = np.random.default_rng(3).normal(size=TC.time_bins + 1)
    g, hist, det = oracle.adjoint(p, TC, n, w_bin=w, w_det=0.4, first_id=11)
    m = oracle.score_moments(p, TC, n, first_id=11)
    assert np.array_equal(m[:, 0], hist.astype(np.float64)) and m[:, 0].sum() == det
    gm = m[:, 1:].T @ w + 0.4 * m[:, 1:].sum(0)
    assert np.allclose(gm, g, rtol=1e-11, atol=0.0)


def _batches(fn, k):
    v = np.array([fn(i) for i in range(k)])
    return v.mean(0), v.std(0, ddof=1) / math.sqrt(k)


def test_tau_score_has_zero_mean_over_detected_photons(oracle):
    p = P.config2()[0]
    n, k = 50_000, 8

    def one(i):
        g, _, _ = oracle.adjoint(p, TC, n, w_det=1.0 / n, first_id=i * n)
        return g[3]

    mean, se = _batches(one, k)
    assert abs(mean) < 4.0 * se, (mean, se)


def test_abs_length_score_matches_crn_fd_of_detected_fraction(oracle):
    """Plain configuration (polished box, absorption only): dD/dLa from the score
    against central differences with the same photons at La (1 +- 2 %)."""
    p = P.config1()[0]
    n, k, rel = 50_000, 8, 0.02
    la = p.abs_length

    def score(i):
        g, _, _ = oracle.adjoint(p, TC, n, w_det=1.0 / n, first_id=i * n)
        return g[0]

    def fd(i):
        up = oracle.adjoint(p.replace(abs_length=la * (1 + rel)), TC, n, first_id=i * n)[2]
        dn = oracle.adjoint(p.replace(abs_length=la * (1 - rel)), TC, n, first_id=i * n)[2]
        return (up - dn) / n / (2 * rel * la)

    gs, es = _batches(score, k)
    gf, ef = _batches(fd, k)
    z = (gs - gf) / math.sqrt(es ** 2 + ef ** 2)
    print("dD/dLa score", gs, "+-", es, "crn fd", gf, "+-", ef, "z", z)
    assert gs > 0 and gf > 0 and abs(z) < 3.0
