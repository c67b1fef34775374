"""The reference project's own GPU callers, relinked against liboptx.so.

oracle/relink.py compiles the reference's tests/test_gpu.cpp and its apps from
the reference sources, with gpu_optical_photons_b200/shim/optx_backend.cpp (the
reference's backend.hpp GPU functions forwarded to the optx C ABI) in place of
the reference's src/gpu/*.cu. These tests run those programs: the reference's
eight GPU test cases must pass unchanged (fast flavour: same-discrete-history
agreement > 99 %; portable flavour: bitwise identity with the reference CPU
build), and the reference's compare / event-bench apps must report agreement.
Without a device the test binary must skip every case and exit 0.
"""
import csv
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RELINK = os.path.join(ROOT, "oracle", "_ref", "relink")


def _exe(flavour, name):
    path = os.path.join(RELINK, flavour, name)
    if not os.path.exists(path):
        pytest.skip("relinked reference programs not built (python oracle/relink.py needs the reference checkout)")
    return path


def _run(cmd, timeout=900):
    return subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)


def _has_gpu():
    import gpu_optical_photons_b200 as g
    return g.gpu_available()


@pytest.mark.parametrize("flavour", ["fast", "portable"])
def test_reference_gpu_tests_skip_without_device(flavour):
    exe = _exe(flavour, "gpu_tests")
    if _has_gpu():
        pytest.skip("a device is present: the GPU test below runs these cases")
    r = _run([exe])
    assert r.returncode == 0, r.stdout + r.stderr
    assert "test cases: 8 | 0 passed | 0 failed | 8 skipped" in r.stdout, r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("flavour", ["fast", "portable"])
def test_reference_gpu_tests_pass(flavour):
    r = _run([_exe(flavour, "gpu_tests")])
    assert r.returncode == 0, r.stdout + r.stderr
    assert "test cases: 8 | 8 passed | 0 failed | 0 skipped" in r.stdout, r.stdout + r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("flavour", ["fast", "portable"])
def test_reference_compare_app(flavour, tmp_path):
    n = 300_000
    r = _run([_exe(flavour, "optphot_compare"), "--n_photons", str(n), "--scat_length", "300",
              "--source", "volume", "--out", str(tmp_path)])
    assert r.returncode == 0, r.stdout + r.stderr
    with open(tmp_path / "compare.json") as f:
        cmp = json.load(f)
    h = cmp["history"]
    assert h["n"] == n
    if flavour == "portable":
        assert h["bitwise_identical"] == n  # exact mode against the portable reference CPU build
    else:
        assert h["fate_differs"] <= 0.001 * n
        assert h["same_discrete"] >= 0.99 * n
    ind = cmp["independent_seed"]
    assert abs(ind["eff_z"]) < 4.0 and ind["time_chi2_p"] > 1e-4 and ind["xy_chi2_p"] > 1e-4


@pytest.mark.gpu
def test_reference_event_bench_app(tmp_path):
    n = 200_003
    out = tmp_path / "event_bench.csv"
    r = _run([_exe("fast", "optphot_event_bench"), "--n_photons", str(n), "--k", "1,4,10000",
              "--repeat", "1", "--csv", str(out), "--surface", "lambertian", "--reflectivity", "0.95",
              "--n_det", "1.5"])
    assert r.returncode == 0, r.stdout + r.stderr
    assert "differs from history-based" not in r.stderr, r.stderr
    with open(out) as f:
        rows = list(csv.DictReader(f))
    hist = [x for x in rows if x["method"] == "history"][0]
    ev = {int(x["k"]): x for x in rows if x["method"] == "event"}
    assert set(ev) == {1, 4, 10000}
    for k, x in ev.items():
        assert int(x["bitwise_identical"]) == n, k
        assert int(x["useful_lane_steps"]) == int(hist["useful_lane_steps"]), k
        assert int(x["issued_lane_steps"]) >= int(x["useful_lane_steps"]), k
    # k >= max_steps: one launch with the history kernel's lane-step accounting
    assert int(ev[10000]["launches"]) == 1
    assert int(ev[10000]["issued_lane_steps"]) == int(hist["issued_lane_steps"])
