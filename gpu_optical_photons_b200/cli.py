"""Command-line runner (the role of the reference's apps/optphot_main.cpp and
apps/optphot_event_bench.cpp): runs one configuration through the history or
the wavefront kernel (or the per-interaction sorted kernels, or gensteps through
the wavefront engine) and prints a JSON line with timings and tallies summary.

    python -m gpu_optical_photons_b200.cli --config config2 --engine wave --n 1e7
    python -m gpu_optical_photons_b200.cli --config config2 --engine sorted --n 1e7
    python -m gpu_optical_photons_b200.cli --config config1 --engine history --mode records --n 1e6

Options mirror the reference's physics keys (--n_det, --abs_length, ...).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import params as P


CONFIGS = {"default": lambda: (P.SimParams(), P.TallyConfig()),
           "config1": P.config1, "config2": P.config2, "config3": P.config3,
           "config3_ref": lambda: P.config3(False)}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--config", default="config1", choices=sorted(CONFIGS))
    ap.add_argument("--engine", default="history", choices=["history", "wave", "sorted", "gensteps"],
                    help="gensteps: --n straight muon tracks through the cube (1 mm gensteps, "
                         "200 photons/mm) expanded into photons by the wavefront engine")
    ap.add_argument("--mode", default="tally", choices=["tally", "records"])
    ap.add_argument("--n", type=float, default=1e6)
    ap.add_argument("--math", default="fast", choices=["fast", "exact", "approx"])
    ap.add_argument("--block", type=int, default=256)
    ap.add_argument("--threshold", type=int, default=28)
    ap.add_argument("--cadence", type=int, default=0)
    ap.add_argument("--bps", type=int, default=0, help="wave engine register budget: 2/3/4 (blocks of "
                    "256) or 7 (blocks of 128); sorted engine: 3 or 4; 0 = default")
    ap.add_argument("--chunk", type=int, default=0)
    ap.add_argument("--host-loop", action="store_true",
                    help="launch waves (sorted: iterations) from the host (no graph)")
    ap.add_argument("--capacity", type=int, default=0,
                    help="sorted engine: photons in flight (default 2^21)")
    ap.add_argument("--repeat", type=int, default=3)
    ap.add_argument("--out", help="write records / tally .npy files and meta.json here "
                    "(the reference's optphot --out layout)")
    ap.add_argument("--time_bins", type=int)
    ap.add_argument("--time_max", type=float)
    ap.add_argument("--xy_bins", type=int)
    for key in ("n_scint", "n_det", "n_out", "abs_length", "scat_length", "reflectivity", "tau",
                "src_x", "src_y", "src_z"):
        ap.add_argument(f"--{key}", type=float)
    ap.add_argument("--surface", choices=sorted(P.SURFACE_NAMES))
    ap.add_argument("--source", choices=["point", "volume"])
    ap.add_argument("--seed", type=int)
    ap.add_argument("--max_steps", type=int)
    a = ap.parse_args(argv)
    if a.repeat < 1:
        ap.error("--repeat must be >= 1")
    if a.engine == "gensteps" and a.mode == "records":
        ap.error("--engine gensteps runs in tally mode only (per-event tallies)")

    import torch
    import gpu_optical_photons_b200 as g
    from .wavefront import WaveConfig, WavefrontEngine

    p, c = CONFIGS[a.config]()
    for key in ("n_scint", "n_det", "n_out", "abs_length", "scat_length", "reflectivity", "tau",
                "src_x", "src_y", "src_z", "seed", "max_steps"):
        v = getattr(a, key)
        if v is not None:
            setattr(p, key, v)
    if a.surface is not None:
        p.surface = P.SURFACE_NAMES[a.surface]
    if a.source is not None:
        p.source = P.POINT if a.source == "point" else P.VOLUME
    for key in ("time_bins", "time_max", "xy_bins"):
        v = getattr(a, key)
        if v is not None:
            setattr(c, key, v)
    n = int(a.n)
    out = {"config": a.config, "engine": a.engine, "mode": a.mode, "n": n, "math": a.math,
           "device": g.gpu_device_name()}
    times = []
    if a.engine == "history":
        if a.mode == "tally":
            dev = torch.zeros(c.length, dtype=torch.int64, device="cuda")
            for _ in range(a.repeat):
                dev.zero_()
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                g.tally_device(p, c, n, out=dev, block_size=a.block, math=a.math)
                torch.cuda.synchronize()
                times.append((time.perf_counter() - t0) * 1e3)
            flat = dev.cpu().numpy().astype(np.uint64)
        else:
            rec = g.device_records(n)
            for _ in range(a.repeat):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                g.records_device(p, n, out=rec, block_size=a.block, math=a.math)
                torch.cuda.synchronize()
                times.append((time.perf_counter() - t0) * 1e3)
            r = g.records_to_numpy(rec)
            flat = None
            out["steps"] = int(r.steps().sum())
            if a.out:
                from . import io
                meta = io.params_to_json(p, io.RunOptions("gpu", "records", n, 1, a.block, c))
                io.write_records(a.out, r, meta)
    elif a.engine == "sorted":
        from .wavefront import SortedEngine
        eng = SortedEngine(a.capacity, 0, a.math, host_loop=a.host_loop, blocks_per_sm=a.bps)
        dev = torch.zeros(c.length, dtype=torch.int64, device="cuda") if a.mode == "tally" else None
        rec = g.device_records(n) if a.mode == "records" else None
        for _ in range(a.repeat):
            if dev is not None:
                dev.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            eng.run(p, n, tally=c if dev is not None else None, tally_out=dev, records_out=rec)
            out["sorted"] = eng.stats()  # synchronises
            times.append((time.perf_counter() - t0) * 1e3)
        eng.close()
        if dev is not None:
            flat = dev.cpu().numpy().astype(np.uint64)
        else:
            r = g.records_to_numpy(rec)
            flat = None
            out["steps"] = int(r.steps().sum())
            if a.out:
                from . import io
                meta = io.params_to_json(p, io.RunOptions("gpu", "records", n, 1, a.block, c))
                io.write_records(a.out, r, meta)
    elif a.engine == "gensteps":
        from . import gensteps as G
        events, gs = G.muon_events(n, seed=p.seed)
        cfg = WaveConfig(block_size=a.block, threshold=a.threshold, cadence=a.cadence,
                         blocks_per_sm=a.bps, chunk=a.chunk, use_graph=not a.host_loop, math=a.math,
                         max_gensteps=len(gs))
        eng = WavefrontEngine(c, len(events), G.photons_of(gs), cfg)
        eng.set_gensteps(events, gs)
        for _ in range(a.repeat):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            eng.run_tally()
            torch.cuda.synchronize()
            times.append((time.perf_counter() - t0) * 1e3)
        tl = eng.tallies()
        out["stats"] = eng.stats()
        out["gensteps"] = len(gs)
        out["photons"] = G.photons_of(gs)
        eng.close()
        flat = None
        out["steps"] = int(tl[:, -2].sum() + tl[:, -1].sum() + tl[:, 1].sum())
        out["fates"] = [int(v) for v in tl[:, :5].sum(0)]
        n = out["photons"]
    else:
        cfg = WaveConfig(block_size=a.block, threshold=a.threshold, cadence=a.cadence,
                         blocks_per_sm=a.bps, chunk=a.chunk, use_graph=not a.host_loop, math=a.math)
        eng = WavefrontEngine(c, 1, n, cfg)
        eng.set_events([p], [n])
        rec = g.device_records(n) if a.mode == "records" else None
        for _ in range(a.repeat):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            if rec is None:
                eng.run_tally()
            else:
                eng.run_records(rec)
            torch.cuda.synchronize()
            times.append((time.perf_counter() - t0) * 1e3)
        out["stats"] = eng.stats()
        if rec is None:
            flat = eng.tallies()[0]
        else:
            r = g.records_to_numpy(rec)
            flat = None
            out["steps"] = int(r.steps().sum())
            if a.out:
                from . import io
                meta = io.params_to_json(p, io.RunOptions("gpu", "records", n, 1, a.block, c))
                io.write_records(a.out, r, meta)
        eng.close()
    if flat is not None:
        t = g.Tally.from_flat(flat, c)
        out["fates"] = [int(v) for v in t.fate_counts]
        out["steps"] = t.steps()
        if a.out:
            from . import io
            meta = io.params_to_json(p, io.RunOptions("gpu", "tally", n, 1, a.block, c))
            io.write_tally(a.out, t, meta)
    best = min(times)
    out["ms"] = best
    out["photons_per_s"] = n / (best * 1e-3)
    out["photon_steps_per_s"] = out["steps"] / (best * 1e-3)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
