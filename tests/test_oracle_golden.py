"""The CPU oracle against the reference's own outputs (golden fixtures made by
tests/golden/make_golden.py from the reference's CPU backend) and against the
Random123 Philox known-answer vectors of the reference's tests/test_rng.cpp."""
import numpy as np
import pytest

from gpu_optical_photons_b200 import params as P
from helpers import compare_histories, golden_records, params_from_meta


def test_philox_known_answers(oracle, golden):
    _, meta = golden
    for kat in meta["philox_kat"]:
        assert list(oracle.philox(kat["ctr"], kat["key"])) == kat["expected"]


def test_stream_is_block_concatenation(oracle, golden):
    # tests/test_rng.cpp:49-57: stream words = Philox blocks {b, 0, id_lo, id_hi}.
    arrays, meta = golden
    sc = meta["stream_case"]
    assert np.array_equal(oracle.stream(sc["seed"], sc["id"], 12), arrays["stream_case/words"])


def test_stream_resume_from_draws(oracle):
    # tests/test_rng.cpp:60-71: resuming after any number of draws continues the stream.
    full = oracle.stream(7, 123456789012, 30)
    for skip in range(13):
        assert np.array_equal(oracle.stream(7, 123456789012, 9, skip=skip), full[skip:skip + 9])


def test_u32_to_uniform_edges(oracle):
    # tests/test_rng.cpp:32-36
    L = oracle.lib()
    assert L.oracle_u32_to_uniform(0) == np.float32(1.0 / 16777216.0)
    assert L.oracle_u32_to_uniform(0xFFFFFFFF) == 1.0
    assert L.oracle_u32_to_uniform(0xFF) == L.oracle_u32_to_uniform(0)


def test_fresnel_normal_incidence(oracle):
    # tests/test_fresnel.cpp:41-42: stilbene / air at normal incidence.
    assert abs(oracle.lib().oracle_fresnel(1.63, 1.0, 1.0) - 0.0573812) < 1e-6
    assert oracle.lib().oracle_fresnel(1.63, 1.63, 0.0) == 0.0          # index matched, grazing
    assert oracle.lib().oracle_fresnel(1.63, 1.0, 0.2) == 1.0           # TIR


def test_fresnel_brewster_and_angle_form(oracle):
    # tests/test_fresnel.cpp:76-96: at Brewster's angle Rp = 0, so R = Rs / 2;
    # over 0.5..89.5 degrees R agrees with the angle-form expressions to 2e-5.
    import math
    f = oracle.lib().oracle_fresnel
    tb = math.atan(1.63 / 1.0)
    tt = math.asin(1.0 / 1.63 * math.sin(tb))
    rs = math.sin(tb - tt) / math.sin(tb + tt)
    assert abs(f(1.0, 1.63, math.cos(tb)) - 0.5 * rs * rs) <= 1e-6

    def angle_form(n1, n2, th):
        s = n1 / n2 * math.sin(th)
        if s >= 1.0:
            return 1.0
        tt = math.asin(s)
        if th == 0.0:
            return ((n1 - n2) / (n1 + n2)) ** 2
        a = math.sin(th - tt) / math.sin(th + tt)
        b = math.tan(th - tt) / math.tan(th + tt)
        return 0.5 * (a * a + b * b)

    for n1, n2 in ((1.63, 1.0), (1.0, 1.63), (1.63, 1.5), (1.5, 1.63)):
        for k in range(1, 180):
            th = math.radians(0.5 * k)
            got = f(n1, n2, float(np.float32(math.cos(th))))
            assert abs(got - angle_form(n1, n2, th)) <= 2e-5, (n1, n2, 0.5 * k, got)


def test_streams_differ_and_are_uniform(oracle):
    # tests/test_rng.cpp:73-118: different photons and seeds give different
    # streams; the first four deviates of 250k consecutive photon streams are
    # uniform (chi2 p > 1e-4, mean within 5 sigma) and neighbouring streams'
    # first deviates are uncorrelated.
    from scipy import stats
    a, b, c = oracle.stream(1, 0, 1000), oracle.stream(1, 1, 1000), oracle.stream(2, 0, 1000)
    assert (a == b).sum() <= 1 and (a == c).sum() <= 1
    n_ph = 250_000
    w = np.stack([oracle.stream(777, i, 4) for i in range(n_ph)])
    u = (((w >> 8) + 1).astype(np.float64) * 2.0 ** -24)
    assert u.min() > 0.0 and u.max() <= 1.0
    n = u.size
    assert abs(u.mean() - 0.5) < 5.0 * np.sqrt(1.0 / 12.0 / n)
    first = u[:, 0] - 0.5
    corr = float((first[1:] * first[:-1]).sum() / n_ph) * 12.0
    assert abs(corr) < 5.0 / np.sqrt(n_ph)
    hist = np.bincount(np.minimum((u.ravel() * 100).astype(int), 99), minlength=100)
    chi2 = float((((hist - n / 100) ** 2) / (n / 100)).sum())
    assert stats.chi2.sf(chi2, 99) > 1e-4


@pytest.mark.parametrize("mode", [0, 1])  # platform (libm) and portable math
def test_rayleigh_cos_inverts_its_cdf(oracle, mode):
    # tests/test_sampling.cpp:90-101: F(mu) = (mu^3 + 3 mu + 4) / 8 inverts the
    # Cardano sampler to 2e-6 on u = i / 1000, mu stays in [-1, 1].
    f = oracle.lib().oracle_rayleigh_cos
    for i in range(1, 1001):
        u = i / 1000.0
        mu = float(f(u, mode))
        assert -1.0 <= mu <= 1.0
        assert abs((mu ** 3 + 3.0 * mu + 4.0) / 8.0 - float(np.float32(u))) <= 2e-6, (u, mu)
    assert abs(float(f(0.5, mode))) <= 1e-7
    assert abs(float(f(1.0, mode)) - 1.0) <= 1e-6


CASES = ["default", "default_scat300_volume", "config1", "config2", "config3_all_specular",
         "black_box", "absorption", "mirror_box", "capped", "big_seed_id"]


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("tag,mode", [("platform", 0), ("portable", 1)])
def test_oracle_reproduces_reference_records(oracle, golden, name, tag, mode):
    arrays, meta = golden
    case = meta["cases"][name]
    p = params_from_meta(case["params"])
    rec = oracle.records(p, case["n"], case["first_id"], mode=mode, threads=2)
    h = compare_histories(rec, golden_records(arrays, name, tag))
    assert h["bitwise_identical"] == case["n"], h


@pytest.mark.parametrize("name", ["config1", "config2"])
@pytest.mark.parametrize("tag,mode", [("platform", 0), ("portable", 1)])
def test_oracle_reproduces_reference_tally(oracle, golden, name, tag, mode):
    arrays, meta = golden
    case = meta["tally_cases"][name]
    p = params_from_meta(case["params"])
    c = P.TallyConfig(case["time_bins"], case["time_max"], case["xy_bins"])
    t = oracle.tally(p, c, case["n"], 0, mode=mode, threads=2)
    assert np.array_equal(t, arrays[f"tally/{name}/{tag}"])


def test_oracle_threads_do_not_change_results(oracle):
    # tests/test_transport_cpu.cpp:313-343 (determinism and first_id tail).
    p = P.SimParams(scat_length=200.0, source=P.VOLUME)
    a = oracle.records(p, 20000, 0, threads=1)
    b = oracle.records(p, 20000, 0, threads=4)
    assert compare_histories(a, b)["bitwise_identical"] == 20000
    tail = oracle.records(p, 500, 1000, threads=1)
    assert np.array_equal(tail["t"], a["t"][1000:1500])
    c = P.TallyConfig()
    t = oracle.tally(p, c, 20000, 0, threads=3)
    counts = np.bincount(a["fate"], minlength=5)
    assert np.array_equal(t[:5], counts)
    assert t[5:5 + c.time_bins + 1].sum() == counts[0]


@pytest.mark.skipif(not __import__("oracle.oracle", fromlist=["x"]).ref_available(),
                    reason="reference CPU backend not built here (oracle/_ref)")
@pytest.mark.parametrize("mode", [0, 1])
def test_oracle_matches_live_reference(oracle, mode):
    """Larger samples against the reference backend compiled from its own sources."""
    for p in (P.config1()[0], P.config2()[0], P.config3(False)[0],
              P.SimParams(scat_length=300.0, source=P.VOLUME, max_steps=7)):
        a = oracle.records(p, 50000, 123, mode=mode)
        b, _ = oracle.ref_records(p, 50000, 123, mode=mode)
        h = compare_histories(a, b)
        assert h["bitwise_identical"] == 50000, h
