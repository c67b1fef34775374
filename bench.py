"""Benchmark of the batched optical-photon transport on B200.

Workload: 4096 events with lognormal photon counts (median 1e4, sigma 1, clamped
to [1e2, 1e6]; 66,481,565 photons, ~2.8e8 photon-steps), per-event absorption
length, reflectivity, refractive index and scattering length, point sources
uniform in a 50 mm cube, Lambertian faces, per-event tallies (100 arrival-time
bins over 0-50 ns + overflow, 10x10 hit map). A step is one run of the whole
batch: one CUDA-graph launch of the persistent wavefront engine.

  value  photon-steps/s with the event table resident on the device
  e2e    photon-steps/s through the C ABI call optx_run_batch with pinned host
         buffers: H2D of the event table and D2H of the per-event tallies inside
         the timed region

``--impl reference`` times the reference's own CPU implementation
(run_cpu_tally of the reference backend, compiled from its sources into
oracle/_ref; the oracle port when that is absent) on the same workload.
Multi-GPU (torchrun): every rank transports its own shard of photons (the same
event list with photon ids offset by rank x photons, so shards are disjoint;
no collective on the data path), value = all ranks' steps / max time over ranks.
The engine settings (register budget, compaction threshold, block size,
cadence, queue depth) come from the autotuner unless given on the command line.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "photon-steps/s (batched wavefront, 4096 events)"
UNIT = "photon-steps/s"
# Algorithmic work per photon-step of this workload: 250.2 scalar ops (91.0 FP32
# arithmetic/compare, 3.63 log/sin/cos/cbrt calls, 155.6 Philox/uniform integer
# ops), counted by the oracle's op-counting scalar type over 64 events x 500
# photons (tests/test_opcount.py checks this constant against the oracle).
OPS_PER_STEP = 250.2
# State-queue bytes per spilled photon: one 64-byte write and one 64-byte read.
QUEUE_BYTES_PER_SPILL = 128
SMS, FP32_LANES_PER_SM = 148, 128


def workload_name(n_events: int) -> str:
    """The benchmarked workload, named identically by both arms."""
    return (f"batched events: {n_events} events, lognormal photons/event (median 1e4, sigma 1, "
            "[1e2,1e6]), Lambertian cube, per-event tallies")


def workload_config(events, counts) -> dict:
    """The `config` of both arms' lines: the workload alone, identical in both
    (what each arm ran per step and its timing details are keys of their own).
    L2: the optx arm writes 256 MB (> the 126 MB L2) between timed steps,
    outside its CUDA events; the reference arm is CPU code."""
    return {"workload": workload_name(len(events)), "events": len(events),
            "photons_per_step": int(np.asarray(counts).sum()),
            "l2": "optx arm: flushed between timed steps (256 MB write, outside the CUDA events); "
                  "reference arm: CPU code (no device cache involved)"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="optx", choices=["optx", "reference"])
    ap.add_argument("--threshold", type=int, default=0, help="0: tuned default")
    ap.add_argument("--block", type=int, default=0)
    ap.add_argument("--bps", type=int, default=0, help="resident blocks per SM (register budget)")
    ap.add_argument("--chunk", type=int, default=0, help="photons a warp claims per grab (0: 256)")
    ap.add_argument("--no-autotune", action="store_true", help="use the default engine settings")
    ap.add_argument("--math", default="fast", choices=["fast", "exact", "approx"],
                    help="math mode of the kernels (see include/optx.h)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the adjoint replay / forward cost measurement")
    ap.add_argument("--no-single-configs", action="store_true",
                    help="skip the single-configuration legs (four setups at their specified sizes)")
    ap.add_argument("--no-compaction", action="store_true",
                    help="skip the forced-compaction leg (state-queue HBM traffic)")
    ap.add_argument("--no-other-math", action="store_true",
                    help="skip timing the same batch in the other two math modes")
    ap.add_argument("--no-history-baseline", action="store_true",
                    help="skip the plain history-kernel baseline (one launch per event)")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the parity check of the benchmarked batch against the reference CPU run")
    ap.add_argument("--no-ksweep", action="store_true",
                    help="skip the history vs forced-compaction (k = 1, 4, 8) records leg")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="reference arm: skip the reference's own GPU kernels (CPU value only)")
    ap.add_argument("--events", type=int, default=4096)
    ap.add_argument("--host-loop", action="store_true",
                    help="launch the waves from the host instead of the graph while loop "
                         "(same kernels; used for per-kernel profiling)")
    return ap.parse_args()


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        backend = "nccl" if args.impl == "optx" else "gloo"
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 100 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int, cmd=None):
        self.index = index
        self.cmd = cmd  # the sampling command (default: nvidia-smi every 100 ms)
        self.proc = None
        self.lines = []
        self.first = threading.Event()

    def __enter__(self):
        cmd = self.cmd or ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                           "--format=csv,noheader,nounits", "-lms", "100"]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # The sampler's start-up can take longer than a short timed region:
            # the region starts once the first sample is in (at most 5 s wait).
            self.first.wait(timeout=5.0)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())
            self.first.set()
        self.first.set()

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def steps_of_tallies(t: np.ndarray) -> int:
    """photon-steps = sum n_boundary + sum n_scatter + absorbed in bulk (per event rows)."""
    t = np.asarray(t, dtype=np.uint64).reshape(-1, t.shape[-1])
    return int(t[:, -2].sum() + t[:, -1].sum() + t[:, 1].sum())


def cpu_reference_leg(events, counts, tc, max_events: int, threads: int = 0, first: int = 0,
                      keep: bool = False):
    """Reference CPU tally (oracle/_ref, the reference's default build) or the
    oracle port over events first .. max_events-1, each event with its photon ids
    offset_i .. offset_i + n_i - 1 (first_id = offset_i). Returns (cpu_baseline
    dict, photon-steps/s, the per-event tallies when keep, else None)."""
    from oracle import oracle as O
    kind = "reference" if O.ref_available() else "port"
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)
    steps = 0
    photons = 0
    rows = []
    t0 = time.perf_counter()
    for i in range(first, max_events):
        if kind == "reference":
            t, _ = O.ref_tally(events[i], tc, int(counts[i]), int(offs[i]), threads=threads)
        else:
            t = O.tally(events[i], tc, int(counts[i]), int(offs[i]), threads=threads)
        steps += steps_of_tallies(t[None, :])
        photons += int(counts[i])
        if keep:
            rows.append(t)
    dt = time.perf_counter() - t0
    cores = (O.ref(0).ref_max_threads() if kind == "reference" else os.cpu_count()) if threads == 0 else threads
    return ({"value": steps / dt, "unit": UNIT, "cores": int(cores), "kind": kind, "photon_steps": steps,
             "sample": f"events {first}..{max_events - 1} of {len(counts)} ({photons} photons, {steps} photon-steps), "
                       f"run_cpu_tally per event, {dt:.1f} s"}, steps / dt,
            np.stack(rows) if keep else None)


def chi2_two_sample(a, b):
    """Two-sample chi-squared of two histograms with different totals (Numerical
    Recipes 14.3, as the reference's include/optphot/stats.hpp): (chi2, ndf, p)."""
    from scipy import stats as ss
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    A, B = a.sum(), b.sum()
    m = (a + b) > 0
    d = np.sqrt(B / A) * a[m] - np.sqrt(A / B) * b[m]
    chi2 = float((d * d / (a[m] + b[m])).sum())
    ndf = int(m.sum()) - 1
    return chi2, ndf, float(ss.chi2.sf(chi2, ndf)) if ndf > 0 else 1.0


def tally_parity(gpu_tallies, cpu_tallies, tc) -> dict:
    """Per-event tallies of the same photons from the GPU and the CPU (rows 0 ..
    len(cpu_tallies) - 1): detected counts, fate-count changes (at least
    sum |delta| / 2 photons changed fate) and the two-sample chi-squared p of the
    summed arrival-time histogram and hit map."""
    ne = len(cpu_tallies)
    g = np.asarray(gpu_tallies[:ne], np.uint64)
    c = np.asarray(cpu_tallies, np.uint64)
    photons = int(c[:, :5].sum())
    d_det = g[:, 0].astype(np.int64) - c[:, 0].astype(np.int64)
    d_fates = int(np.abs(g[:, :5].astype(np.int64) - c[:, :5].astype(np.int64)).sum())
    t0, x0 = 5, 5 + tc.time_bins + 1
    _, _, p_time = chi2_two_sample(g[:, t0:x0].sum(axis=0), c[:, t0:x0].sum(axis=0))
    _, _, p_hit = chi2_two_sample(g[:, x0:x0 + tc.xy_bins ** 2].sum(axis=0), c[:, x0:x0 + tc.xy_bins ** 2].sum(axis=0))
    return {"events": ne, "photons": photons,
            "detected_gpu": int(g[:, 0].sum()), "detected_cpu": int(c[:, 0].sum()),
            "abs_delta_detected_over_photons": int(np.abs(d_det).sum()) / photons,
            "fate_count_changes_lower_bound_frac": d_fates / 2 / photons,
            "chi2_p_time_hist": p_time, "chi2_p_hit_map": p_hit,
            "total_photons_equal": int(g[:, :5].sum()) == photons}


def parity_leg(gpu_tallies, cpu_tallies, events, counts, tc, cfg, math: str, k_records: int = 64) -> dict:
    """The benchmarked batch against the reference CPU run of the same photons.

    Tallies (events 0 .. len(cpu_tallies) - 1): detected counts, per-event fate
    counts (at least sum |delta| / 2 photons changed fate) and the two-sample
    chi-squared p of the summed arrival-time histogram and hit map. Records
    (events 0 .. k_records - 1): the same engine variant in batched records mode
    against the reference CPU's records, photon by photon (fate and discrete
    history agreement, the reference's compare_histories)."""
    import torch
    from oracle import oracle as O
    from gpu_optical_photons_b200.backend import device_records, records_to_numpy
    from gpu_optical_photons_b200.wavefront import WavefrontEngine
    out = {**tally_parity(gpu_tallies, cpu_tallies, tc), "gpu_math": math,
           "cpu": "reference run_cpu_tally (default build)" if O.ref_available() else "oracle port (default math)"}
    p_time, p_hit = out["chi2_p_time_hist"], out["chi2_p_hit_map"]
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)
    k = min(k_records, len(events))
    m = int(offs[k])
    eng = WavefrontEngine(tc, k, m, cfg)
    try:
        eng.set_events(events[:k], counts[:k])
        d = device_records(m)
        eng.run_records(d)
        torch.cuda.synchronize()
        rec = records_to_numpy(d)
        del d
    finally:
        eng.close()
    same_fate = same_disc = 0
    for i in range(k):
        lo, hi = int(offs[i]), int(offs[i + 1])
        if O.ref_available():
            r, _ = O.ref_records(events[i], hi - lo, lo)
        else:
            r = O.records(events[i], hi - lo, lo)
        f = rec["fate"][lo:hi] == r["fate"]
        same_fate += int(f.sum())
        same_disc += int((f & (rec["n_boundary"][lo:hi] == r["n_boundary"])
                          & (rec["n_scatter"][lo:hi] == r["n_scatter"])).sum())
    out["records"] = {"events": k, "photons": m, "fate_agreement": same_fate / m,
                      "same_discrete_history": same_disc / m}
    out["pass"] = bool(out["abs_delta_detected_over_photons"] <= 1e-3 and p_time > 0.01 and p_hit > 0.01
                       and out["records"]["fate_agreement"] >= 0.999 and out["total_photons_equal"])
    return out


def history_baseline(g, events, counts, tc, first_id: int, math: str, stream, reps: int = 2):
    """The batch as the plain history kernel runs it: one optx_tally_device launch
    per event, back to back on one stream (the reference's way to process many
    events: one run_gpu_tally each), timed with CUDA events after one warm-up
    pass. Returns (photon-steps/s, ms per pass, tallies of the last pass)."""
    import torch
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    dev = torch.zeros((len(events), tc.length), dtype=torch.int64, device="cuda")
    sptr = stream.cuda_stream
    rows = [dev[i] for i in range(len(events))]  # contiguous rows of tc.length: checked by construction

    def one_pass():
        dev.zero_()
        for i, e in enumerate(events):
            if counts[i]:
                g.tally_device(e, tc, int(counts[i]), first_id=first_id + int(offs[i]), out=rows[i],
                               math=math, stream=sptr, check=False)

    one_pass()
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        one_pass()
        b.record(stream)
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    t = dev.cpu().numpy().astype(np.uint64)
    m = float(np.median(ms))
    return steps_of_tallies(t) / (m * 1e-3), m, t


def adjoint_cost(math: str, n: int = 10_000_000, reps: int = 5) -> dict:
    """Cost of the path-replay adjoint against one forward run on the calibration
    setup (the Lambertian cube with Rayleigh scattering and a volume source at
    theta = (La 1000, Ls 700, R 0.95, tau 4), 1e7 photons, 500 arrival-time bins):
    median CUDA-event times of the forward tally and of the replay that
    accumulates dLoss/dtheta (both the bare C-ABI run, no host read-back inside
    the events), and of the common-random-number central finite
    differences the adjoint replaces (two forward runs per parameter, at
    theta_j (1 +- 1e-3), parameter upload included)."""
    import torch
    from gpu_optical_photons_b200.adjoint import ResponseModel
    from gpu_optical_photons_b200.params import TallyConfig, config2
    from gpu_optical_photons_b200.wavefront import WaveConfig
    base = config2()[0]
    theta = (1000.0, 700.0, 0.95, 4.0)
    tcal = TallyConfig(500, 50.0, 1)
    m = ResponseModel(base, n, tcal, config=WaveConfig(math=math))
    try:
        w = torch.ones(tcal.time_bins + 1, dtype=torch.float64)
        m.forward(theta)
        m.replay(theta, w, 0.5)
        from gpu_optical_photons_b200 import _lib
        wd = w.cuda()
        gd = torch.zeros(4, dtype=torch.float64, device="cuda")
        st = torch.cuda.current_stream().cuda_stream

        def replay_run():
            _lib.call("optx_engine_run_adjoint", m.engine._h, ctypes.c_void_p(wd.data_ptr()), 0.5,
                      ctypes.c_void_p(gd.data_ptr()), ctypes.c_void_p(st))

        mom = torch.empty((tcal.time_bins + 1) * 5, dtype=torch.float64, device="cuda")

        def moments_run():
            _lib.call("optx_engine_run_score_moments", m.engine._h, ctypes.c_void_p(mom.data_ptr()),
                      ctypes.c_void_p(st))

        # The loss's gradient in one pass: the score-moment replay gives the
        # histogram h and its Jacobian J = dE[h]/dtheta from the same photons, so
        # the loss (Poisson NLL of h against a target, plus the detected
        # fraction D = sum h / n) and its gradient J^T dL/dh + sum_b J_b / n come
        # from one run; the host does the 500 x 4 product.
        target = np.asarray(m.forward((800.0, 600.0, 0.93, 3.5))[0], np.float64)
        m._upload(theta)
        moments_run()
        torch.cuda.synchronize()

        def one_pass_gradient():
            moments_run()
            M = mom.view(tcal.time_bins + 1, 5).cpu().numpy()   # synchronises
            h, J = M[:, 0], M[:, 1:]
            lam = h[:tcal.time_bins] + 1.0
            dl_dh = np.zeros_like(h)
            dl_dh[:tcal.time_bins] = (1.0 - target[:tcal.time_bins] / lam) / n
            dl_dh += 1.0 / n                                      # dD/dh_b
            loss = float((lam - target[:tcal.time_bins] * np.log(lam)).sum() / n + h.sum() / n)
            return loss, J.T @ dl_dh

        def forward_loss():
            m.engine.run_tally()
            flat = m.engine.tallies()                            # synchronises
            h = flat[0, 5:5 + tcal.time_bins + 1].astype(np.float64)
            lam = h[:tcal.time_bins] + 1.0
            return float((lam - target[:tcal.time_bins] * np.log(lam)).sum() / n + h.sum() / n)

        fwd, adj, fd, one, one_wall, fwd_wall = [], [], [], [], [], []
        for _ in range(reps):
            m._upload(theta)  # back at theta after the FD runs (outside the timed regions)
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(); m.engine.run_tally(); b.record(); torch.cuda.synchronize()
            fwd.append(a.elapsed_time(b))
            a.record(); replay_run(); b.record(); torch.cuda.synchronize()
            adj.append(a.elapsed_time(b))
            a.record()
            for j in range(4):
                for sgn in (1.0, -1.0):
                    th = list(theta)
                    th[j] = theta[j] * (1.0 + sgn * 1e-3)
                    m._upload(th)
                    m.engine.run_tally()
            b.record(); torch.cuda.synchronize()
            fd.append(a.elapsed_time(b))
            m._upload(theta)
            torch.cuda.synchronize()
            a.record(); moments_run(); b.record(); torch.cuda.synchronize()
            one.append(a.elapsed_time(b))
            t0 = time.perf_counter(); one_pass_gradient(); one_wall.append((time.perf_counter() - t0) * 1e3)
            t0 = time.perf_counter(); forward_loss(); fwd_wall.append((time.perf_counter() - t0) * 1e3)
        # The one-pass gradient equals the replay of dL/dh (same photons).
        loss, g1 = one_pass_gradient()
        lam = np.asarray(m.forward(theta)[0])[:tcal.time_bins] + 1.0
        wb = torch.zeros(tcal.time_bins + 1, dtype=torch.float64)
        wb[:tcal.time_bins] = torch.from_numpy((1.0 - target[:tcal.time_bins] / lam) / n)
        g2 = m.replay(theta, wb, 1.0 / n)
        agree = float(np.max(np.abs(g1 - g2) / np.maximum(np.abs(g2), 1e-300)))
    finally:
        m.close()
    f, r, c = float(np.median(fwd)), float(np.median(adj)), float(np.median(fd))
    o, ow, fw = float(np.median(one)), float(np.median(one_wall)), float(np.median(fwd_wall))
    return {"forward_ms": f, "replay_ms": r, "replay_over_forward": r / f,
            "crn_fd_ms": c, "adjoint_over_crn_fd": (f + r) / c, "photons": n,
            "one_pass": {"moments_ms": o, "over_forward": o / f,
                         "gradient_wall_ms": ow, "forward_loss_wall_ms": fw, "wall_over_forward": ow / fw,
                         "max_rel_diff_vs_replay_gradient": agree,
                         "what": "loss and its gradient from one score-moment replay (histogram + Jacobian, "
                                 "J^T dL/dh on the host) against one forward run; wall times include the "
                                 "read-back of the tally / moment table and the host arithmetic"},
            "what": "adjoint = one forward + one replay; CRN FD = 8 forward runs (2 per parameter)",
            "setup": "Lambertian cube, Rayleigh, volume source, theta=(1000, 700, 0.95, 4), 500 time bins"}


def compaction_leg(events, counts, tc, first_id, cfg, stream, tallies, hbm_peak, reps: int = 3,
                   cadence: int = 8) -> dict:
    """The same batch with a forced compaction every `cadence` steps per wave (the
    reference event kernel's k steps per launch): live photons go through the
    state queues (64 B written + 64 B read per spill), so this leg measures the
    queues' HBM traffic. Tallies are checked equal to the one-wave run's."""
    import torch
    from dataclasses import replace
    from gpu_optical_photons_b200.wavefront import WavefrontEngine
    n_photons = int(counts.sum())
    e2 = WavefrontEngine(tc, len(events), n_photons, replace(cfg, cadence=cadence))
    try:
        sptr = stream.cuda_stream
        e2.set_events(events, counts, first_id, stream=sptr)
        e2.run_tally(stream=sptr)
        torch.cuda.synchronize()
        ms = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream); e2.run_tally(stream=sptr); b.record(stream); torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        st = e2.stats(stream=sptr)
        assert np.array_equal(e2.tallies(stream=sptr), tallies), "compacted run's tallies differ"
    finally:
        e2.close()
    t = float(np.median(ms))
    qb = QUEUE_BYTES_PER_SPILL * int(st["spills"])
    return {"cadence": cadence, "ms_per_step": t, "value": steps_of_tallies(tallies) / (t * 1e-3),
            "waves": int(st["launches"]), "spills": int(st["spills"]), "queue_bytes": qb,
            "queue_gbs": qb / (t * 1e-3) / 1e9, "hbm_peak_gbs": hbm_peak,
            "queue_frac_of_hbm": qb / (t * 1e-3) / 1e9 / hbm_peak,
            "what": "queue bytes = 128 B per spilled photon (4 x 16 B stores + 4 x 16 B loads)"}


def run_reference(args):
    # The reference is a CPU code: rank 0 alone runs it; other ranks exit at once.
    if int(os.environ.get("RANK", "0")) != 0:
        return
    from gpu_optical_photons_b200.params import TallyConfig
    from gpu_optical_photons_b200.wavefront import batched_events
    events, counts = batched_events(n_events=args.events)
    tc = TallyConfig(100, 50.0, 10)
    # Warm-up steps run a 256-event slice (thread pool, page faults); every timed
    # step runs the whole batch, the workload of the optx arm's value.
    warm = min(256, len(events))
    for s in range(args.warmup):
        cpu_reference_leg(events, counts, tc, warm)
    vals, secs = [], []
    base = None
    for s in range(args.steps):
        t0 = time.perf_counter()
        base, v, _ = cpu_reference_leg(events, counts, tc, len(events))
        secs.append(time.perf_counter() - t0)
        vals.append(v)
    value = float(np.median(vals))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.median(secs)) * 1e3,
            "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded event generator)",
            "config": workload_config(events, counts),
            "per_step": "the whole batch: run_cpu_tally per event (all host threads)",
            "warmup_steps": f"{warm}-event slice",
            "photon_steps_per_step": base["photon_steps"],
            "cpu_baseline": {**base, "value": value,
                             "sample": "the whole batch per step; " + base["sample"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not args.no_reference_gpu:
        rg = reference_gpu_leg(events, counts, tc)
        if rg is not None:
            line["reference_gpu"] = rg
        rs = reference_gpu_single_configs()
        if rs is not None:
            line["reference_gpu_single_configs"] = rs
        rk = reference_gpu_ksweep()
        if rk is not None:
            line["reference_gpu_ksweep"] = rk
    print(json.dumps(line), flush=True)


def single_setups():
    """The single configurations at their specified sizes: (name, params, tally,
    photons). The polished cube (1e6 photons), the wrapped-Lambertian cube with
    Rayleigh scattering (1e8), the long bar with its black -z face (1e8; per-face
    surfaces, which the reference cannot express) and the same bar with all side
    and end faces specular (1e8; the reference-compatible variant)."""
    from gpu_optical_photons_b200.params import config1, config2, config3
    return [("polished_cube", *config1(), 1_000_000),
            ("wrapped_lambertian_rayleigh", *config2(), 100_000_000),
            ("long_bar_black_minus_z", *config3(True), 100_000_000),
            ("long_bar_specular", *config3(False), 100_000_000)]


def _ev_ms(fn, reps: int) -> float:
    """Median CUDA-event time of fn on the current stream after one warm-up call."""
    import torch
    fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(); fn(); b.record(); torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    return float(np.median(ts))


def single_config_legs(math: str, reps: int = 3) -> dict:
    """One configuration at its specified size (single_setups(), tally mode): the
    wavefront engine (host-call settings: 7 blocks of 128 threads), the
    per-interaction sorted kernels (photons queued in HBM by pending
    interaction, one launch per iteration) and this library's history kernel.
    Median CUDA-event kernel times; the three tallies are checked equal. (The
    reference's own kernels on the same workloads are timed by the reference
    arm, `--impl reference`.)"""
    import torch
    from gpu_optical_photons_b200 import backend as B
    from gpu_optical_photons_b200.wavefront import SortedEngine, WaveConfig, WavefrontEngine
    ev_ms = lambda fn: _ev_ms(fn, reps)  # noqa: E731

    out = {}
    for name, p, c, n in single_setups():
        eng = WavefrontEngine(c, 1, n, WaveConfig(blocks_per_sm=7, math=math))
        try:
            eng.set_events([p], [n])
            wave = ev_ms(eng.run_tally)
            t = eng.tallies()[0]
        finally:
            eng.close()
        steps = int(t[-2] + t[-1] + t[1])
        dev = torch.zeros(c.length, dtype=torch.int64, device="cuda")

        def hist_run():
            dev.zero_()
            B.tally_device(p, c, n, out=dev, math=math)
        hist = ev_ms(hist_run)
        ht = dev.cpu().numpy().astype(np.uint64)
        srt = SortedEngine(math=math)
        try:
            def sorted_run():
                dev.zero_()
                srt.run(p, n, tally=c, tally_out=dev)
            sorted_ms = ev_ms(sorted_run)
            sst = srt.stats()
            stt = dev.cpu().numpy().astype(np.uint64)
        finally:
            srt.close()
        assert np.array_equal(ht, t) and np.array_equal(stt, t), f"{name}: tallies differ between kernels"
        out[name] = {"photons": n, "photon_steps": steps, "wavefront_ms": wave, "history_ms": hist,
                     "sorted_ms": sorted_ms, "sorted_iterations": sst["iterations"],
                     "wavefront_photon_steps_per_s": steps / (wave * 1e-3),
                     "history_photon_steps_per_s": steps / (hist * 1e-3),
                     "wavefront_over_history": hist / wave, "tallies_equal": True}
    return out


def ksweep_leg(math: str, n: int = 10_000_000, reps: int = 3) -> dict:
    """The wrapped-Lambertian cube with Rayleigh scattering (1e7 photons, records
    mode) as the reference's event benchmark runs it (apps/optphot_event_bench.cpp:
    130-143): the history kernel against the wavefront engine with a forced
    compaction every k steps (k = 1, 4, 8: the reference event kernel's steps
    per launch) and with none (one wave), records checked bit-identical across
    all runs. Median CUDA-event kernel times (host read-back excluded). The
    reference's own kernels on the same workload are the reference arm's
    `reference_gpu_ksweep`."""
    import torch
    from gpu_optical_photons_b200 import backend as B
    from gpu_optical_photons_b200.params import config2
    from gpu_optical_photons_b200.wavefront import WaveConfig, WavefrontEngine
    p, c = config2()
    d = B.device_records(n)
    hist = _ev_ms(lambda: B.records_device(p, n, out=d, math=math), reps)
    torch.cuda.synchronize()
    want = {k: v.clone() for k, v in d.items()}
    steps = int((want["n_boundary"].long().sum() + want["n_scatter"].long().sum()
                 + (want["fate"] == 1).long().sum()).item())
    out = {"photons": n, "photon_steps": steps, "history_ms": hist, "wavefront": {}}
    for k in (0, 1, 4, 8):
        eng = WavefrontEngine(c, 1, n, WaveConfig(blocks_per_sm=7, math=math, cadence=k))
        try:
            eng.set_events([p], [n])
            ms = _ev_ms(lambda: eng.run_records(d), reps)
            st = eng.stats()
        finally:
            eng.close()
        torch.cuda.synchronize()
        same = all(torch.equal(d[f], want[f]) for f in d)
        assert same, f"records differ at cadence {k}"
        out["wavefront"]["one_wave" if k == 0 else f"k{k}"] = {
            "ms": ms, "waves": int(st["launches"]), "spills": int(st["spills"]),
            "photon_steps_per_s": steps / (ms * 1e-3), "records_bitwise_equal_history": True}
    del d, want
    torch.cuda.empty_cache()
    return out


def reference_gpu_leg(events, counts, tc):
    """The same batch through the reference's own GPU backend rebuilt for sm_100a
    (oracle/_ref/libref_gpu.so: src/gpu/gpu_backend.cu compiled by nvcc from the
    reference sources): one run_gpu_tally call per event, as the reference's API
    processes events (each call allocates, launches, copies back and frees).
    Informational, beside the CPU value; None without the library or a GPU."""
    from oracle import oracle as O
    try:
        import torch
        if not (O.refgpu_available() and torch.cuda.is_available()):
            return None
    except Exception:
        return None
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)

    def one_pass():
        steps, kms = 0, 0.0
        t0 = time.perf_counter()
        for i, e in enumerate(events):
            if counts[i]:
                t, tm = O.refgpu_tally(e, tc, int(counts[i]), int(offs[i]))
                steps += steps_of_tallies(t[None, :])
                kms += tm["kernel_ms"]
        return steps, (time.perf_counter() - t0) * 1e3, kms

    one_pass()  # warm-up: context, module load, clocks
    steps, wall_ms, kms = one_pass()
    return {"value": steps / (wall_ms * 1e-3), "unit": UNIT, "ms_per_step": wall_ms,
            "kernel_only_value": steps / (kms * 1e-3), "kernel_ms_per_step": kms, "calls": int((counts > 0).sum()),
            "what": "reference src/gpu/gpu_backend.cu built for sm_100a from its sources; run_gpu_tally per event "
                    "(host buffers, allocation per call), same 4096-event batch and tally binning"}


def reference_gpu_single_configs(reps: int = 3):
    """The reference's tally kernel (rebuilt for sm_100a) on the single
    configurations the optx arm's `single_configs` key times that the reference
    can express (every one but the long bar's black -z face): median kernel time
    reported by its run_gpu_tally. None without the library or a GPU."""
    from oracle import oracle as O
    try:
        import torch
        if not (O.refgpu_available() and torch.cuda.is_available()):
            return None
    except Exception:
        return None
    out = {}
    for name, p, c, n in single_setups():
        if p.faces_c() is not None:  # per-face surfaces: not expressible in the reference
            continue
        O.refgpu_tally(p, c, n)  # warm-up
        runs = [O.refgpu_tally(p, c, n) for _ in range(reps)]
        t = runs[0][0]
        steps = steps_of_tallies(t[None, :])
        kms = float(np.median([tm["kernel_ms"] for _, tm in runs]))
        out[name] = {"photons": n, "photon_steps": steps, "kernel_ms": kms,
                     "kernel_photon_steps_per_s": steps / (kms * 1e-3)}
    return out


def reference_gpu_ksweep(n: int = 10_000_000, reps: int = 3):
    """The reference's records kernels (rebuilt for sm_100a) on the optx arm's
    `ksweep` workload (wrapped-Lambertian cube, 1e7 photons): run_gpu_records
    (history kernel) and run_gpu_records_event with k = 1, 4, 8 steps per launch
    (compaction between launches); median kernel times as the reference reports
    them (its event kernels' sum, host loop excluded). None without the library
    or a GPU."""
    from oracle import oracle as O
    try:
        import torch
        if not (O.refgpu_available() and torch.cuda.is_available()):
            return None
    except Exception:
        return None
    from gpu_optical_photons_b200.params import config2
    p, _ = config2()
    O.refgpu_records(p, n)  # warm-up
    runs = [O.refgpu_records(p, n) for _ in range(reps)]
    r0 = runs[0][0]
    steps = int(r0["n_boundary"].astype(np.int64).sum() + r0["n_scatter"].astype(np.int64).sum()
                + (r0["fate"] == 1).sum())
    out = {"photons": n, "photon_steps": steps,
           "history_kernel_ms": float(np.median([tm["kernel_ms"] for _, tm in runs])), "event": {}}
    for k in (1, 4, 8):
        O.refgpu_records_event(p, n, k)  # warm-up
        ev = [O.refgpu_records_event(p, n, k) for _ in range(reps)]
        out["event"][f"k{k}"] = {"kernels_ms": float(np.median([st["kernels_ms"] for _, st, _ in ev])),
                                 "total_ms": float(np.median([tm["total_ms"] for _, _, tm in ev])),
                                 "launches": ev[0][1]["launches"]}
    return out


def run_optx(args):
    import torch
    world, rank, local, pg = dist_setup(args)
    torch.cuda.set_device(local)
    from gpu_optical_photons_b200 import build
    build.build()
    import gpu_optical_photons_b200 as g
    from gpu_optical_photons_b200 import _lib
    from gpu_optical_photons_b200.params import CSimParams, TallyConfig
    from gpu_optical_photons_b200.wavefront import WaveConfig, WavefrontEngine, batched_events
    from gpu_optical_photons_b200.distributed import max_over_ranks, shard_first_id

    events, counts = batched_events(n_events=args.events)
    n_photons = int(counts.sum())
    first_id = shard_first_id(rank, n_photons)  # disjoint photon ids per rank
    tc = TallyConfig(100, 50.0, 10)
    cfg = WaveConfig(block_size=args.block or 256, threshold=args.threshold or 28,
                     blocks_per_sm=args.bps or 3, use_graph=not args.host_loop, math=args.math,
                     chunk=args.chunk)
    tuned = None
    if not args.no_autotune and not args.host_loop and not (args.threshold or args.bps or args.block or args.chunk):
        from gpu_optical_photons_b200.autotune import tune
        t0 = time.perf_counter()
        cfg, tune_log = tune(events, counts, tc, base=cfg, repeats=2)
        tuned = {"seconds": round(time.perf_counter() - t0, 1), "candidates": len(tune_log)}
    eng = WavefrontEngine(tc, len(events), n_photons, cfg)
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream

    # Pinned host buffers for the e2e leg.
    arr = (CSimParams * len(events))(*[e.to_c() for e in events])
    ev_pinned = torch.empty(ctypes.sizeof(arr), dtype=torch.uint8, pin_memory=True)
    ctypes.memmove(ev_pinned.data_ptr(), ctypes.addressof(arr), ctypes.sizeof(arr))
    cnt_pinned = torch.from_numpy(counts.astype(np.int64)).pin_memory()
    out_pinned = torch.empty((len(events), tc.length), dtype=torch.int64, pin_memory=True)
    h2d_bytes = len(events) * 112 + (len(events) + 1) * 8 + 256   # DevParams table + offsets + run args
    d2h_bytes = len(events) * tc.length * 8 + 64                  # tallies + control block

    eng.set_events(events, counts, first_id, stream=sptr)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    # warm-up
    for _ in range(args.warmup):
        eng.run_tally(stream=sptr)
    torch.cuda.synchronize()
    st0 = eng.stats(stream=sptr)
    tallies = eng.tallies(stream=sptr)
    steps_per_run = steps_of_tallies(tallies)
    assert int(tallies[:, :5].sum()) == n_photons

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t_wall = time.perf_counter()
        for k in range(args.steps):
            flush.zero_()                       # L2 flush between timed steps (outside the events)
            starts[k].record(stream)
            eng.run_tally(stream=sptr)
            ends[k].record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t_wall
    if pg:
        pg.barrier()
    dev_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    ms_step = sum(dev_ms) / args.steps
    st = eng.stats(stream=sptr)
    waves = int(st["launches"])
    if pg:
        ms_step = max_over_ranks(ms_step, pg, device="cuda")
    value = world * steps_per_run / (ms_step * 1e-3)

    # e2e: the C ABI call with host buffers (H2D table, run, D2H tallies) per step.
    L = _lib.lib()
    sts = _lib.CEventStats()
    tmg = _lib.CTiming()
    e2e_ms = []
    for k in range(args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _lib.check(L.optx_run_batch(eng._h, ctypes.c_void_p(ev_pinned.data_ptr()), None,
                                    ctypes.c_void_p(cnt_pinned.data_ptr()), len(events), first_id,
                                    ctypes.c_void_p(out_pinned.data_ptr()), ctypes.byref(sts),
                                    ctypes.byref(tmg)))
        dt = (time.perf_counter() - t0) * 1e3
        if k >= args.warmup:
            e2e_ms.append(dt)
    e2e_step = float(np.mean(e2e_ms))
    if pg:
        e2e_step = max_over_ranks(e2e_step, pg, device="cuda")
    assert np.array_equal(out_pinned.numpy().astype(np.uint64), tallies)

    clocks = clk.summary()
    peak_mhz = clocks["sm_max_mhz"] or 1965.0
    peak_gops = SMS * FP32_LANES_PER_SM * peak_mhz * 1e6 / 1e9
    achieved_gops = OPS_PER_STEP * steps_per_run / (ms_step * 1e-3) / 1e9
    # DRAM bytes (read + write) of the wave kernel over one run of this batch,
    # from an ncu capture of the benchmarked batch itself (profiles/); the
    # tallies, event records and queues it moves scale with events, not steps,
    # so only a capture of the same batch gives the per-step figure.
    traffic = None
    prof = os.path.join(HERE, "profiles", "wave_kernel_batched.json")
    if os.path.exists(prof):
        with open(prof) as f:
            pj = json.load(f)
        if pj.get("events") == len(events) and pj.get("photons") == n_photons:
            traffic = pj.get("dram_bytes_per_run")
    queue_bytes = QUEUE_BYTES_PER_SPILL * int(st["spills"])
    peaks = {}
    peaks_path = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        with open(peaks_path) as f:
            peaks = json.load(f)
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    hbm_src = ("measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks
               else "fallback 6650 GB/s (no MEASURED_PEAKS.json)")

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded event generator)",
        "config": workload_config(events, counts),
        "photon_steps_per_step": steps_per_run,
        "photons_per_s": world * n_photons / (ms_step * 1e-3),
        "parallelism": f"dp{world} (independent event batches per GPU)",
        "autotune": tuned,
        "engine": {"block_size": cfg.launch_block_size, "threshold": cfg.threshold,
                   "wave_quota": cfg.wave_quota,
                   "blocks_per_sm": cfg.blocks_per_sm,
                   "cadence": cfg.cadence, "chunk": cfg.chunk or 256,
                   "tail_steps": cfg.tail_steps or 4096,
                   "graph": cfg.use_graph, "math": cfg.math},
        "e2e": {"value": world * steps_per_run / (e2e_step * 1e-3), "unit": UNIT,
                "h2d_bytes_per_step": h2d_bytes, "d2h_bytes_per_step": d2h_bytes,
                "ms_per_step": e2e_step, "call": "optx_run_batch (pinned host buffers)"},
        "gpu_launches": args.steps * (waves + 1),
        "waves_per_step": waves,
        "simt_efficiency": st["simt_efficiency"],
        "roofline": {"bound": "issue", "achieved": achieved_gops, "peak": peak_gops, "unit": "Gop/s",
                     "frac": achieved_gops / peak_gops, "traffic": traffic,
                     "peak_source": f"nominal FP32 lane issue rate {SMS} SMs x {FP32_LANES_PER_SM} lanes x "
                                    f"{peak_mhz:.0f} MHz (max SM clock seen); no measured issue peak exists",
                     "ops_per_photon_step": OPS_PER_STEP,
                     "hbm": {"queue_bytes_per_step": queue_bytes,
                             "achieved_gbs": queue_bytes / (ms_step * 1e-3) / 1e9,
                             "peak_gbs": hbm_peak,
                             "frac": queue_bytes / (ms_step * 1e-3) / 1e9 / hbm_peak,
                             "peak_source": hbm_src}},
        "clocks": clocks,
        "wall_s_timed": wall,
    }
    if not args.no_other_math:
        # The same batch and engine settings in the other math modes (EXACT: bitwise
        # parity with the reference CPU build; APPROX: hardware transcendental units).
        from dataclasses import replace
        other = {}
        for m in ("fast", "exact", "approx"):
            if m == args.math:
                continue
            e2 = WavefrontEngine(tc, len(events), n_photons, replace(cfg, math=m))
            e2.set_events(events, counts, first_id, stream=sptr)
            for _ in range(args.warmup):
                e2.run_tally(stream=sptr)
            torch.cuda.synchronize()
            ms = []
            for _ in range(min(args.steps, 20)):
                flush.zero_()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                e2.run_tally(stream=sptr)
                b.record(stream)
                torch.cuda.synchronize()
                ms.append(a.elapsed_time(b))
            t2 = e2.tallies(stream=sptr)
            e2.close()
            mm = float(np.mean(ms))
            if pg:
                mm = max_over_ranks(mm, pg, device="cuda")
            other[m] = {"value": world * steps_of_tallies(t2) / (mm * 1e-3), "ms_per_step": mm,
                        "photon_steps_per_step": steps_of_tallies(t2)}
        line["other_math_modes"] = other
    if not args.no_adjoint:
        line["adjoint"] = adjoint_cost(args.math)
    if not args.no_single_configs:
        line["single_configs"] = single_config_legs(args.math)
    if not args.no_compaction:
        line["compaction_leg"] = compaction_leg(events, counts, tc, first_id, cfg, stream, tallies,
                                                hbm_peak)
    if not args.no_history_baseline:
        hv, hms, ht = history_baseline(g, events, counts, tc, first_id, args.math, stream)
        # Same per-photon arithmetic, integer tallies: the two engines agree exactly.
        assert np.array_equal(ht, tallies), "history and wavefront tallies differ"
        line["history_baseline"] = {
            "value": world * hv, "unit": UNIT, "ms_per_step": hms, "launches": len(events),
            "what": "one history-kernel launch (optx_tally_device) per event, back to back on one "
                    "stream; identical tallies checked",
            "speedup_of_value": value / (world * hv)}
    if not args.no_ksweep:
        line["ksweep"] = ksweep_leg(args.math)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:  # the CPU baseline is an N=1 figure
        # All host threads on events 0..1023, then one thread on events 0..255
        # (the reference's threads = n and threads = 1, apps/optphot_bench.cpp:125-158).
        base, _, cpu_t = cpu_reference_leg(events, counts, tc, max_events=min(1024, len(events)),
                                           keep=not args.no_parity and first_id == 0)
        one, _, _ = cpu_reference_leg(events, counts, tc, max_events=min(256, len(events)), threads=1)
        base["single_thread"] = one
        line["cpu_baseline"] = base
        if cpu_t is not None:
            line["parity"] = parity_leg(tallies, cpu_t, events, counts, tc, cfg, args.math)
    if rank == 0:
        print(json.dumps(line), flush=True)
    eng.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_optx(a)
