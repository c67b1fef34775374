"""Autotuner of the wavefront engine.

Chooses, for a given workload (a batch of events with their photon counts and
a tally configuration), the engine settings by measurement on the device:

* ``blocks_per_sm`` — the register budget of the wave kernel as resident blocks
  per SM (2, 3 or 4 blocks of 256 threads: <= 128 / 80 / 64 registers; 7 blocks
  of 128 threads: <= 72 registers);
* ``threshold`` — refill a warp when fewer than this many lanes are alive (the
  compaction threshold: higher keeps warps fuller, lower refills less often);
* ``block_size`` — threads per block;
* ``cadence`` — forced compaction after this many steps in a wave (0 = only when
  the wave's work runs out);
* ``chunk`` — consecutive photons a warp claims with one atomic (larger keeps a
  warp on one event longer, so its shared-memory tally slots hit more often;
  smaller balances the end of a wave better);
* ``tail_steps`` — steps a photon makes in a wave before the end-of-wave
  compaction may move it to the next wave (large: warps keep their photons
  until they finish, one wave per run);
* ``wave_quota`` — fresh photons admitted per wave, i.e. the depth of the work
  queue between two compactions (0 = all photons in the first wave).

Staged coordinate search: (blocks_per_sm x threshold) first, then block size,
cadence, chunk, tail steps and queue depth around the best point. Each candidate is timed with
CUDA events on the launching stream (median of `repeats` runs after one warm-up
run), on the real workload. Every candidate computes the same tallies (the
engine's results do not depend on these settings), which `tune` checks.

`tune_sorted` does the same for the per-interaction sorted kernels of one
configuration: register budget (3 or 4 blocks of 256 threads per SM) x queue
capacity (photons in flight), exhaustively; the best budget differs between
workloads (the divergent Lambertian cube prefers 4, the long specular bar 3).
"""
from __future__ import annotations

import itertools
import json
import time
from dataclasses import asdict, replace

import numpy as np

from .params import TallyConfig
from .wavefront import SortedEngine, WaveConfig, WavefrontEngine


def time_config(cfg: WaveConfig, events, counts, tally: TallyConfig, repeats: int = 3,
                first_id: int = 0):
    """(median ms per run, tallies, stats) of one engine configuration."""
    import torch
    eng = WavefrontEngine(tally, len(events), int(np.sum(counts)), cfg)
    try:
        eng.set_events(events, counts, first_id)
        eng.run_tally()  # warm-up: graph instantiation, caches
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ms = []
        for _ in range(repeats):
            s.record()
            eng.run_tally()
            e.record()
            torch.cuda.synchronize()
            ms.append(s.elapsed_time(e))
        return float(np.median(ms)), eng.tallies(), eng.stats()
    finally:
        eng.close()


def tune(events, counts, tally: TallyConfig, base: WaveConfig | None = None, repeats: int = 3,
         bps=(2, 3, 4, 7), thresholds=(16, 20, 24, 28, 32), blocks=(128, 256), cadences=(0, 32),
         quota_fracs=(0.0, 0.25), chunks=(64, 256, 1024), tails=(64, 4096), verbose: bool = False):
    """Returns (best WaveConfig, list of measurement dicts)."""
    base = base or WaveConfig()
    total = int(np.sum(counts))
    log = []
    ref_tallies = None

    def measure(cfg):
        nonlocal ref_tallies
        t0 = time.perf_counter()
        ms, tallies, st = time_config(cfg, events, counts, tally, repeats)
        if ref_tallies is None:
            ref_tallies = tallies
        elif not np.array_equal(tallies, ref_tallies):
            raise AssertionError(f"engine settings changed the tallies: {cfg}")
        rec = {**asdict(cfg), "ms": ms, "simt": st["simt_efficiency"], "waves": st["launches"],
               "tune_s": time.perf_counter() - t0}
        log.append(rec)
        if verbose:
            print(json.dumps(rec), flush=True)
        return ms

    best_cfg, best_ms = None, float("inf")
    for b, t in itertools.product(bps, thresholds):
        cfg = replace(base, blocks_per_sm=b, threshold=t)
        ms = measure(cfg)
        if ms < best_ms:
            best_cfg, best_ms = cfg, ms
    for bs in blocks:
        if bs == best_cfg.block_size or best_cfg.blocks_per_sm == 7:  # 7 implies 128-thread blocks
            continue
        cfg = replace(best_cfg, block_size=bs)  # same register budget, smaller blocks
        ms = measure(cfg)
        if ms < best_ms:
            best_cfg, best_ms = cfg, ms
    for c in cadences:
        if c == best_cfg.cadence:
            continue
        cfg = replace(best_cfg, cadence=c)
        ms = measure(cfg)
        if ms < best_ms:
            best_cfg, best_ms = cfg, ms
    for ch in chunks:
        if ch == (best_cfg.chunk or 256):
            continue
        cfg = replace(best_cfg, chunk=ch)
        ms = measure(cfg)
        if ms < best_ms:
            best_cfg, best_ms = cfg, ms
    for tl in tails:
        if tl == (best_cfg.tail_steps or 4096):
            continue
        cfg = replace(best_cfg, tail_steps=tl)
        ms = measure(cfg)
        if ms < best_ms:
            best_cfg, best_ms = cfg, ms
    for f in quota_fracs:
        q = int(total * f)
        if q == best_cfg.wave_quota:
            continue
        cfg = replace(best_cfg, wave_quota=q)
        ms = measure(cfg)
        if ms < best_ms:
            best_cfg, best_ms = cfg, ms
    return best_cfg, log


def tune_sorted(p, tally: TallyConfig, n: int, budgets=(3, 4),
                capacities=(1 << 20, 1 << 21, 1 << 22), repeats: int = 3, math="fast"):
    """Best (blocks_per_sm, capacity) of the sorted kernels for n photons of the
    configuration p, by CUDA-event timing (median of `repeats` after a warm-up
    run). Returns (best, table) with table[(blocks_per_sm, capacity)] = ms;
    raises if two candidates give different tallies."""
    import torch
    table, ref = {}, None
    for bps, cap in itertools.product(budgets, capacities):
        eng = SortedEngine(cap, 0, math, blocks_per_sm=bps)
        try:
            out = torch.zeros(tally.length, dtype=torch.int64, device="cuda")

            def run():
                out.zero_()
                eng.run(p, n, tally=tally, tally_out=out)

            run()
            eng.stats()  # warm-up; raises on a failed run
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ms = []
            for _ in range(repeats):
                s.record()
                run()
                e.record()
                torch.cuda.synchronize()
                ms.append(s.elapsed_time(e))
            eng.stats()
        finally:
            eng.close()
        t = out.cpu().numpy()
        if ref is None:
            ref = t
        elif not np.array_equal(t, ref):
            raise RuntimeError(f"sorted run at blocks_per_sm={bps}, capacity={cap} changed the tally")
        table[(bps, cap)] = float(np.median(ms))
    best = min(table, key=table.get)
    return {"blocks_per_sm": best[0], "capacity": best[1]}, table


def main(argv=None):
    import argparse
    from .wavefront import batched_events
    ap = argparse.ArgumentParser(description="tune the wavefront engine on the batched workload")
    ap.add_argument("--events", type=int, default=4096)
    ap.add_argument("--repeats", type=int, default=3)
    a = ap.parse_args(argv)
    events, counts = batched_events(n_events=a.events)
    best, log = tune(events, counts, TallyConfig(100, 50.0, 10), repeats=a.repeats, verbose=True)
    print(json.dumps({"best": asdict(best), "ms": min(r["ms"] for r in log)}))


if __name__ == "__main__":
    main()
