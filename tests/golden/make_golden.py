"""Generates the golden fixtures in tests/golden/ from the reference itself.

Run in a checkout where the reference (zmeskma/GPU_Optical_photons) is
available and oracle/Makefile has built oracle/_ref (``make -C oracle ref``):

    python tests/golden/make_golden.py

It writes, for each case below, the records of photons first_id .. first_id+n-1
produced by the reference's own run_cpu_records (src/cpu/cpu_backend.cpp) in
the default build (platform libm) and in the OPTPHOT_PORTABLE_MATH build, plus
run_cpu_tally outputs, into golden_records.npz. The Philox known-answer vectors
are the Random123 ones of the reference's tests/test_rng.cpp:24-30, read from
that file as text. The GPU box never runs this script; tests read the .npz.
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from gpu_optical_photons_b200 import params as P  # noqa: E402
from oracle import oracle as O  # noqa: E402

REFERENCE = O.reference_root()

CASES = {
    # name: (SimParams, n, first_id)
    "default": (P.SimParams(), 3000, 0),
    "default_scat300_volume": (P.SimParams(scat_length=300.0, source=P.VOLUME), 3000, 1000),
    "config1": (P.config1()[0], 3000, 0),
    "config2": (P.config2()[0], 3000, 5),
    "config3_all_specular": (P.config3(False)[0], 2000, 0),
    "black_box": (P.black_box().replace(src_x=10.0, src_y=-5.0, src_z=3.0), 3000, 0),
    "absorption": (P.black_box().replace(abs_length=100.0, src_x=6.0, src_y=-8.0, src_z=-5.0), 3000, 0),
    "mirror_box": (P.SimParams(surface=P.SPECULAR, reflectivity=1.0, n_det=1.0, abs_length=P.INF,
                               max_steps=1000, src_x=3.0, src_y=-11.0, src_z=7.0, seed=5), 1000, 0),
    "capped": (P.SimParams(scat_length=300.0, max_steps=5), 3000, 0),
    "big_seed_id": (P.SimParams(scat_length=300.0, seed=0x0123456789ABCDEF), 2000, (1 << 40) + 17),
}

TALLY_CASES = {
    "config1": (P.config1()[0], P.config1()[1], 20000),
    "config2": (P.config2()[0], P.config2()[1], 20000),
}


def kat_vectors():
    """Philox KAT triples (ctr, key, expected) from the reference's test_rng.cpp, as text."""
    src = open(os.path.join(REFERENCE, "tests", "test_rng.cpp")).read()
    calls = re.findall(r"check_kat\(\s*\{([^}]*)\},\s*\{([^}]*)\},\s*\{([^}]*)\}\)", src, re.S)
    out = []
    for ctr, key, exp in calls:
        parse = lambda s: [int(v.strip().rstrip("u"), 16) for v in s.split(",")]
        out.append({"ctr": parse(ctr), "key": parse(key), "expected": parse(exp)})
    return out


def main():
    O.build(with_ref=True)
    arrays = {}
    meta = {"cases": {}, "tally_cases": {}}
    for name, (p, n, first_id) in CASES.items():
        for mode, tag in ((O.PLATFORM, "platform"), (O.PORTABLE, "portable")):
            rec, _ = O.ref_records(p, n, first_id, mode=mode)
            for k in O.Records.FIELDS:
                arrays[f"{name}/{tag}/{k}"] = rec[k]
        meta["cases"][name] = {"n": n, "first_id": first_id,
                               "params": {f[0]: getattr(p, f[0]) for f in P.CSimParams._fields_}}
    for name, (p, c, n) in TALLY_CASES.items():
        for mode, tag in ((O.PLATFORM, "platform"), (O.PORTABLE, "portable")):
            t, _ = O.ref_tally(p, c, n, 0, mode=mode)
            arrays[f"tally/{name}/{tag}"] = t
        meta["tally_cases"][name] = {"n": n, "time_bins": c.time_bins, "time_max": c.time_max,
                                     "xy_bins": c.xy_bins,
                                     "params": {f[0]: getattr(p, f[0]) for f in P.CSimParams._fields_}}
    kats = kat_vectors()
    assert len(kats) == 3, kats
    meta["philox_kat"] = kats
    # The reference's PhiloxStream concatenation case (test_rng.cpp:49-57): the stream
    # of (seed, id) is blocks {b, 0, id_lo, id_hi} of the reference's own philox4x32_10.
    seed, pid = 0x0123456789ABCDEF, 0xFEDCBA9876543210
    meta["stream_case"] = {"seed": seed, "id": pid}
    key = [seed & 0xFFFFFFFF, seed >> 32]
    words = [O.ref_philox([b, 0, pid & 0xFFFFFFFF, pid >> 32], key) for b in range(3)]
    arrays["stream_case/words"] = np.concatenate(words).astype(np.uint32)
    for k, v in meta["cases"].items():
        v["params"] = {kk: (float(vv) if isinstance(vv, float) else int(vv)) for kk, vv in v["params"].items()}
    for k, v in meta["tally_cases"].items():
        v["params"] = {kk: (float(vv) if isinstance(vv, float) else int(vv)) for kk, vv in v["params"].items()}
    np.savez_compressed(os.path.join(HERE, "golden_records.npz"), **arrays)
    with open(os.path.join(HERE, "golden_meta.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True, default=float)
    print("wrote", len(arrays), "arrays")


if __name__ == "__main__":
    main()
