"""bench.py's reference arm on the CPU: one JSON line with the keys the
benchmark contract asks for, and, under a multi-rank launch, output from rank 0
only (the other ranks exit at once without work)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                           "--steps", "1", "--warmup", "0", "--events", "16"],
                          capture_output=True, text=True, env=env, timeout=600, cwd=ROOT)


def test_reference_arm_prints_one_contract_line(oracle):
    if not oracle.ref_available():
        pytest.skip("the reference's CPU backend is not built here")
    out = _run({})
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "photon-steps/s"
    assert d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] == 0
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    # Both arms name the same workload: the optx arm's `config` is built by the
    # same function from the same events (its line carries run details as
    # keys of their own), so the two configs are equal.
    sys.path.insert(0, ROOT)
    import bench
    from gpu_optical_photons_b200.wavefront import batched_events
    events, counts = batched_events(n_events=16)
    assert d["config"] == bench.workload_config(events, counts)
    assert d["photon_steps_per_step"] == cb["photon_steps"] > 0


def test_reference_arm_other_ranks_exit_quietly():
    out = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert out.returncode == 0, out.stderr[-2000:]
    assert not [l for l in out.stdout.splitlines() if l.startswith("{")]


def test_tally_parity_metrics():
    """bench.py's parity metrics on planted tallies (CPU): equal tallies give no
    differences and p = 1; photons moved from detected to absorbed show up as
    detection and fate-count differences; a shifted arrival-time histogram fails
    the chi-squared test."""
    sys.path.insert(0, ROOT)
    import numpy as np
    import bench
    from gpu_optical_photons_b200 import params as P
    tc = P.TallyConfig(20, 50.0, 2)
    rng = np.random.default_rng(1)
    cpu = np.zeros((6, tc.length), np.uint64)
    for row in cpu:
        fates = rng.multinomial(10_000, [0.6, 0.2, 0.2, 0.0, 0.0])
        row[:5] = fates
        row[5:5 + 21] = rng.multinomial(int(fates[0]), [1 / 21] * 21)
        row[26:30] = rng.multinomial(int(fates[0]), [0.25] * 4)
    same = bench.tally_parity(cpu.copy(), cpu, tc)
    assert same["photons"] == 60_000 and same["total_photons_equal"]
    assert same["abs_delta_detected_over_photons"] == 0 and same["fate_count_changes_lower_bound_frac"] == 0
    assert same["chi2_p_time_hist"] == pytest.approx(1.0) and same["chi2_p_hit_map"] == pytest.approx(1.0)
    moved = cpu.copy()
    moved[0, 0] -= 30
    moved[0, 1] += 30
    moved[0, 5] -= 30  # those photons leave the time histogram and the hit map
    moved[0, 26] -= 30
    d = bench.tally_parity(moved, cpu, tc)
    assert d["abs_delta_detected_over_photons"] == pytest.approx(30 / 60_000)
    assert d["fate_count_changes_lower_bound_frac"] == pytest.approx(30 / 60_000)
    assert d["total_photons_equal"]
    shifted = cpu.copy()
    moved_n = np.minimum(shifted[:, 6], 200)  # photons of the second time bin ...
    shifted[:, 6] -= moved_n
    shifted[:, 5] += moved_n                   # ... counted in the first
    assert bench.tally_parity(shifted, cpu, tc)["chi2_p_time_hist"] < 0.01


def test_clock_sampler_waits_for_its_first_sample(tmp_path):
    """The clock sampler's first sample is in before the timed region starts (a
    sampler slower to start than a short timed region would otherwise record
    nothing), and active throttle reasons are reported by name."""
    import time
    sys.path.insert(0, ROOT)
    import bench
    fake = tmp_path / "smi.sh"
    fake.write_text("#!/bin/bash\nsleep 0.3\nwhile true; do "
                    "echo '0, 1800, 1965, 900.0, Active, Not Active, Not Active, Not Active, Active'; "
                    "sleep 0.05; done\n")
    fake.chmod(0o755)
    with bench.ClockSampler(0, cmd=[str(fake)]) as clk:
        n_at_start = len(clk.lines)
        time.sleep(0.2)
    s = clk.summary()
    assert n_at_start >= 1
    assert s["samples"] >= 1 and s["sm_mhz"] == 1800.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
