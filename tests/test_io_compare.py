"""Output files and the comparison harness against the reference's own code.

The package's `io` (.npy + meta.json) and `compare` (history / distribution
agreement and their JSON) are checked byte for byte against the reference's
src/core/io.cpp, config.cpp and compare.cpp, compiled from the reference
sources into oracle/_ref (ref_write_records, ref_write_tally,
ref_params_to_json, ref_compare_json), on records from the oracle.
"""
import os

import numpy as np
import pytest

from gpu_optical_photons_b200 import compare as C
from gpu_optical_photons_b200 import io as IO
from gpu_optical_photons_b200 import params as P
from gpu_optical_photons_b200.backend import Tally

pytestmark = pytest.mark.usefixtures("oracle")


def _need_ref(oracle):
    if not oracle.ref_available(oracle.PLATFORM):
        pytest.skip("reference CPU build (oracle/_ref) not present")


PARAMS = {
    "default": P.SimParams(),
    "config2": P.config2()[0],
    "config3": P.config3(False)[0],
    "odd": P.SimParams(hx=12.3456789, hy=7.1, hz=0.3, n_scint=1.58123, abs_length=P.INF,
                       scat_length=333.333, surface=P.SPECULAR, reflectivity=0.987654321,
                       source=P.VOLUME, src_x=-1.25e-3, src_y=3.0e7, tau=0.0, max_steps=7, seed=2**63 + 5),
}


@pytest.mark.parametrize("name", list(PARAMS))
def test_meta_json_matches_reference(oracle, name):
    _need_ref(oracle)
    p = PARAMS[name]
    o = IO.RunOptions(backend="gpu", mode="tally", n_photons=123456789, threads=0, block_size=128,
                      tally=P.TallyConfig(500, 37.5, 33))
    got = IO.params_to_json(p, o)
    ref = oracle.ref_params_to_json(p, "gpu", "tally", 123456789, 0, 128, 500, 37.5, 33)
    assert got == ref


def _files(d):
    return sorted(os.listdir(d))


def test_records_files_byte_identical(oracle, tmp_path):
    _need_ref(oracle)
    p = P.config2()[0]
    rec = oracle.records(p, 20_000, 3, mode=oracle.PLATFORM)
    meta = IO.params_to_json(p)
    IO.write_records(str(tmp_path / "ours"), rec, meta)
    oracle.ref_write_records(str(tmp_path / "ref"), rec, meta)
    assert _files(tmp_path / "ours") == _files(tmp_path / "ref")
    for f in _files(tmp_path / "ref"):
        assert (tmp_path / "ours" / f).read_bytes() == (tmp_path / "ref" / f).read_bytes(), f
    back = IO.read_records(str(tmp_path / "ref"))
    for k in rec.FIELDS:
        assert np.array_equal(back[k], rec[k]), k
        assert np.array_equal(np.load(tmp_path / "ours" / f"{k}.npy"), rec[k]), k
    assert IO.read_meta(str(tmp_path / "ours"))["surface"] == "lambertian"


@pytest.mark.parametrize("bins", [(100, 50), (7, 1), (500, 3)])
def test_tally_files_byte_identical(oracle, tmp_path, bins):
    _need_ref(oracle)
    p = P.config2()[0]
    c = P.TallyConfig(bins[0], 50.0, bins[1])
    flat = oracle.tally(p, c, 30_000, 0, mode=oracle.PLATFORM)
    t = Tally.from_flat(flat, c)
    IO.write_tally(str(tmp_path / "ours"), t, "{}")
    oracle.ref_write_tally(str(tmp_path / "ref"), c, flat, "{}")
    for f in _files(tmp_path / "ref"):
        assert (tmp_path / "ours" / f).read_bytes() == (tmp_path / "ref" / f).read_bytes(), f
    back = IO.read_tally(str(tmp_path / "ref"))
    assert np.array_equal(back.fate_counts, t.fate_counts)
    assert np.array_equal(back.time_hist, t.time_hist)
    assert np.array_equal(back.xy_hist, t.xy_hist)
    assert np.load(tmp_path / "ours" / "xy_hist.npy").shape == (bins[1], bins[1])


def test_npy_header_padding():
    for shape in [(0,), (1,), (10**9,), (3, 4), (12345, 6789)]:
        h = IO.npy_bytes_header("<f4", shape)
        assert len(h) % 64 == 0 and h.endswith(b"\n")


def _json_pair(a, b, p, **kw):
    h = C.compare_histories(a, b) if len(a["fate"]) == len(b["fate"]) else None
    d = C.compare_distributions(a, b, p, **kw)
    return (C.history_json(h) if h else "null"), C.distribution_json(d)


@pytest.mark.parametrize("case", ["same_seed_modes", "independent", "identical", "bins_tmax", "sizes"])
def test_compare_json_matches_reference(oracle, case):
    _need_ref(oracle)
    p = P.SimParams(scat_length=300.0, source=P.VOLUME)
    n = 50_000
    a = oracle.records(p, n, 0, mode=oracle.PLATFORM)
    kw = {}
    if case == "same_seed_modes":
        b = oracle.records(p, n, 0, mode=oracle.DOUBLE)  # an FP64 transport: rare decision flips
    elif case == "independent":
        q = P.SimParams(scat_length=300.0, source=P.VOLUME, seed=p.seed + 1)
        b = oracle.records(q, n, 0, mode=oracle.PLATFORM)
    elif case == "identical":
        b = a
    elif case == "bins_tmax":
        b = oracle.records(p, n, 7, mode=oracle.PLATFORM)
        kw = {"time_bins": 37, "t_max": 3.5, "xy_bins": 9}
    else:
        b = oracle.records(p, n // 3, 1, mode=oracle.PLATFORM)
    got = _json_pair(a, b, p, **kw)
    ref = oracle.ref_compare_json(a, b, p, **kw)
    assert got == ref


def test_compare_counts_planted_divergence(oracle):
    p = P.SimParams(scat_length=300.0)
    a = oracle.records(p, 5000, 0, mode=oracle.PLATFORM)
    b = oracle.Records({k: v.copy() for k, v in a.items()})
    b["fate"][17] = (b["fate"][17] + 1) % 5
    b["t"][20] = np.nextafter(b["t"][20], np.float32(np.inf))
    h = C.compare_histories(a, b)
    assert (h.n, h.fate_differs, h.same_discrete, h.bitwise_identical, h.first_divergent) == \
           (5000, 1, 4999, 4998, 17)
    assert h.max_abs_dt > 0


def test_compare_command_on_reference_directories(oracle, tmp_path, capsys):
    """`python -m gpu_optical_photons_b200.compare` on two directories the
    reference's write_records produced prints the reference's comparison JSON."""
    _need_ref(oracle)
    import json
    p = P.config2()[0]
    meta = oracle.ref_params_to_json(p, "cpu", "records", 20_000, 1, 256, 100, 50.0, 50)
    a = oracle.ref_records(p, 20_000, 0, mode=oracle.PLATFORM)[0]
    b = oracle.ref_records(p, 20_000, 0, mode=oracle.PORTABLE)[0]
    oracle.ref_write_records(str(tmp_path / "a"), a, meta)
    oracle.ref_write_records(str(tmp_path / "b"), b, meta)
    assert C.main([str(tmp_path / "a"), str(tmp_path / "b"), "--xy_bins", "25"]) == 0
    got = json.loads(capsys.readouterr().out)
    h, d = oracle.ref_compare_json(a, b, p, 100, 0.0, 25)
    assert got == {"history": json.loads(h), "distribution": json.loads(d)}
    assert C.params_from_meta(IO.read_meta(str(tmp_path / "a"))).to_c().abs_length == p.abs_length


@pytest.mark.gpu
def test_cli_records_out_against_reference_cpu(oracle, tmp_path):
    """GPU records written by the CLI (--out) against the reference CPU build's
    own files for the same seed: the reference's comparison finds >= 99.9 % of
    fates equal and independent-seed-level statistical agreement."""
    _need_ref(oracle)
    import json
    import subprocess
    import sys
    n = 400_000
    d_gpu = tmp_path / "gpu"
    r = subprocess.run([sys.executable, "-m", "gpu_optical_photons_b200.cli", "--config", "default",
                        "--mode", "records", "--n", str(n), "--scat_length", "300", "--source", "volume",
                        "--repeat", "1", "--out", str(d_gpu)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    p = P.SimParams(scat_length=300.0, source=P.VOLUME)
    cpu = oracle.ref_records(p, n, 0, mode=oracle.PLATFORM)[0]
    oracle.ref_write_records(str(tmp_path / "cpu"), cpu, oracle.ref_params_to_json(p, "cpu", "records", n))
    out = subprocess.run([sys.executable, "-m", "gpu_optical_photons_b200.compare", str(tmp_path / "cpu"),
                          str(d_gpu)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    res = json.loads(out.stdout)
    assert res["history"]["n"] == n
    assert res["history"]["fate_differs"] <= 0.001 * n
    assert abs(res["distribution"]["eff_z"]) < 4.0
    assert IO.read_meta(str(d_gpu))["backend"] == "gpu"


@pytest.mark.gpu
@pytest.mark.parametrize("argv", [
    ["--config", "config2", "--engine", "history", "--n", "2e5"],
    ["--config", "config3", "--engine", "wave", "--n", "2e5", "--bps", "7"],
    ["--config", "config1", "--engine", "wave", "--n", "2e5", "--cadence", "8", "--host-loop"],
    ["--engine", "gensteps", "--n", "16"],
    ["--config", "config2", "--engine", "sorted", "--n", "2e5", "--capacity", "8192"],
    ["--config", "config3", "--engine", "sorted", "--n", "2e5", "--host-loop", "--bps", "4"],
])
def test_cli_engines_print_a_consistent_line(engine, capsys, tmp_path, argv):
    """Every engine of the command-line runner prints one JSON line whose fates
    add up to the photons it ran (and, with --out, writes a tally the reader
    gives back)."""
    import json
    from gpu_optical_photons_b200 import cli
    out_dir = tmp_path / "t"
    gs = "gensteps" in argv
    cli.main(argv + ["--repeat", "2"] + ([] if gs else ["--out", str(out_dir)]))
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    n = line.get("photons", line["n"])
    assert sum(line["fates"]) == n and line["steps"] > 0 and line["ms"] > 0
    if not gs:
        t = IO.read_tally(str(out_dir))
        assert int(np.asarray(t.fate_counts).sum()) == n


@pytest.mark.gpu
def test_cli_wave_records_equal_history_records(engine, capsys, tmp_path):
    """--engine wave --mode records writes the engine's per-photon records, which
    equal the history kernel's bit for bit (exact math)."""
    import json
    from gpu_optical_photons_b200 import cli
    base = ["--config", "config2", "--mode", "records", "--n", "50000", "--math", "exact", "--repeat", "1"]
    cli.main(base + ["--engine", "wave", "--out", str(tmp_path / "w")])
    cli.main(base + ["--engine", "history", "--out", str(tmp_path / "h")])
    lines = [json.loads(l) for l in capsys.readouterr().out.strip().splitlines()]
    assert lines[0]["steps"] == lines[1]["steps"] > 0
    w, h = IO.read_records(str(tmp_path / "w")), IO.read_records(str(tmp_path / "h"))
    for k in ("fate", "n_boundary", "n_scatter", "t", "x", "y", "z", "path"):
        assert np.array_equal(np.asarray(w[k]).view(np.uint8), np.asarray(h[k]).view(np.uint8)), k


@pytest.mark.parametrize("argv", [["--engine", "gensteps", "--mode", "records"], ["--repeat", "0"]])
def test_cli_rejects_unsupported_options(argv, capsys):
    """Options the runner cannot honour end with a usage error before any GPU work."""
    from gpu_optical_photons_b200 import cli
    with pytest.raises(SystemExit) as ei:
        cli.main(argv)
    assert ei.value.code == 2
    assert "error" in capsys.readouterr().err


def test_records_resize_replaces_unusable_fields():
    """run_gpu_records writes n entries through each field's pointer, so a
    caller's Records is resized first (the reference resizes the caller's
    vectors): short, long, strided, read-only or wrongly typed fields are
    replaced; fields already fit for n entries are kept as they are."""
    from gpu_optical_photons_b200.backend import Records
    n = 10
    r = Records.empty(n)
    keep = r["t"]
    r["fate"] = np.zeros(3, np.uint8)                       # too short
    r["n_boundary"] = np.zeros(20, np.uint32)               # too long
    r["x"] = np.zeros(2 * n, np.float32)[::2]               # strided
    ro = np.zeros(n, np.float32)
    ro.flags.writeable = False
    r["y"] = ro                                              # read-only
    r["z"] = np.zeros(n, np.float64)                         # wrong type
    del r["path"]                                            # missing
    r.resize(n)
    assert r["t"] is keep
    for k in Records.FIELDS:
        v = r[k]
        assert v.shape == (n,) and v.dtype == Records.DTYPES[k] and v.flags.c_contiguous and v.flags.writeable
