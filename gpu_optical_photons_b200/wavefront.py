"""The wavefront engine (optx_engine_* of include/optx.h) and batched events.

A ``WavefrontEngine`` owns its device state queues, control block, per-event
tallies and captured CUDA graphs. ``set_events`` uploads a batch (one or
thousands of events with their own SimParams and photon counts); the run is
one graph launch: a prep kernel, then a device-side while loop of persistent
wave kernels. Event i owns photon ids ``first_id + offset_i + k``, so each
event reproduces the reference's ``run_cpu_*(p_i, n_i, ..., first_id=offset_i)``.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from .params import (CSimParams, CFaces, LAMBERTIAN, POINT, SimParams, TallyConfig)
from .backend import Tally, _stream_ptr, _crec_from_torch, check_records_out, check_tally_out


@dataclass
class WaveConfig:
    block_size: int = 256
    blocks_per_sm: int = 0      # register budget: 2/3/4 blocks of 256 (128/80/64 regs), 7 blocks of 128 (72); 0 = 3
    threshold: int = 28         # refill when fewer lanes than this are alive
    cadence: int = 0            # forced spill after this many steps per wave (0 = off)
    wave_quota: int = 0         # fresh photons per wave (0 = all)
    use_graph: bool = True
    math: str = "fast"
    chunk: int = 0              # consecutive photons a warp claims per grab (0 = 256)
    max_gensteps: int = 0       # capacity for set_gensteps (0 = no gensteps)
    tail_steps: int = 0         # steps in a wave before a photon may move to the next (0 = 4096)

    @property
    def launch_block_size(self) -> int:
        """Threads per block of the launches: the 72-register budget (7 blocks
        per SM) runs 128-thread blocks when the default 256 is given."""
        return 128 if self.blocks_per_sm == 7 and self.block_size == 256 else self.block_size

    def to_c(self) -> _lib.CWaveConfig:
        return _lib.CWaveConfig(self.launch_block_size, self.blocks_per_sm, self.threshold, self.cadence,
                                self.wave_quota, 1 if self.use_graph else -1, _lib.MATH[self.math],
                                self.chunk, self.max_gensteps, self.tail_steps, 0)


class EventTable:
    """Events converted once to the C layout (optx_params, and optx_faces when any
    event has per-face surfaces), for batches uploaded many times: every
    WavefrontEngine call that takes a list of events also takes an EventTable,
    and skips the per-event Python conversion (about 2 us per event)."""

    def __init__(self, events):
        self.arr, self.faces = _events_c(list(events))
        self.n = len(self.arr)

    def __len__(self):
        return self.n


def _counts_c(counts, n_events: int) -> np.ndarray:
    """Photon counts as the C ABI reads them: one uint64 per event (the call
    reads n_events entries through the pointer)."""
    cnt = np.ascontiguousarray(counts, dtype=np.uint64)
    if cnt.ndim != 1 or cnt.shape[0] != n_events:
        raise ValueError(f"counts must hold one photon count per event ({n_events}), got shape {cnt.shape}")
    return cnt


def _events_c(events):
    if isinstance(events, EventTable):
        return events.arr, events.faces
    arr = (CSimParams * len(events))()
    faces = None
    if any(isinstance(e, SimParams) and e.faces_c() is not None for e in events):
        faces = (CFaces * len(events))()
    for i, e in enumerate(events):
        arr[i] = e.to_c() if isinstance(e, SimParams) else e
        if faces is not None:
            f = e.faces_c() if isinstance(e, SimParams) else None
            if f is None:  # this event uses one surface model on all five faces
                f = CFaces((ctypes.c_uint32 * 6)(*([e.surface] * 6)),
                           (ctypes.c_float * 6)(*([e.reflectivity] * 6)))
            faces[i] = f
    return arr, faces


class WavefrontEngine:
    def __init__(self, tally: TallyConfig, max_events: int = 1, max_photons: int = 1 << 24,
                 config: WaveConfig | None = None):
        self.tally_config = tally
        self.config = config or WaveConfig()
        self.max_events = max_events
        self.max_photons = max_photons
        self._h = ctypes.c_void_p()
        cc = tally.to_c()
        wc = self.config.to_c()
        _lib.call("optx_engine_create", ctypes.byref(cc), max_events, max_photons, ctypes.byref(wc),
                  ctypes.byref(self._h))
        self.n_events = 0
        self.counts = None

    def close(self):
        if self._h:
            _lib.lib().optx_engine_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_events(self, events, counts, first_id: int = 0, stream=0):
        """Uploads a batch; `events` is a list of SimParams (or CSimParams)."""
        arr, faces = _events_c(events)
        cnt = _counts_c(counts, len(arr))
        self._keep = (arr, faces, cnt)
        _lib.call("optx_engine_set_events", self._h, ctypes.cast(arr, ctypes.c_void_p),
                  ctypes.cast(faces, ctypes.c_void_p) if faces is not None else None,
                  cnt.ctypes.data, len(events), first_id, ctypes.c_void_p(stream or 0))
        self.n_events = len(events)
        self.counts = cnt

    def set_gensteps(self, events, gensteps, first_id: int = 0, stream=0):
        """Uploads gensteps (a GENSTEP_DTYPE array, see gensteps.py) emitting into
        `events` (their physics and tally slices); tallies() then has one row per event."""
        from .gensteps import as_gensteps
        arr, faces = _events_c(events)
        g = as_gensteps(gensteps)
        self._keep = (arr, faces, g)
        _lib.call("optx_engine_set_gensteps", self._h, ctypes.cast(arr, ctypes.c_void_p),
                  ctypes.cast(faces, ctypes.c_void_p) if faces is not None else None, len(events),
                  g.ctypes.data, len(g), first_id, ctypes.c_void_p(stream or 0))
        self.n_events = len(events)
        self.counts = np.bincount(g["event"], weights=g["n_photons"], minlength=len(events)).astype(np.uint64)

    def set_gensteps_device(self, events, dev_gensteps, first_id: int = 0, stream=0):
        """Uploads gensteps that are already in device memory (a CUDA tensor of
        optx_genstep records, 40 bytes each, e.g. from gensteps.to_device): the
        records and photon offsets are built on the device, asynchronously on
        `stream`. Invalid gensteps are reported by the next tallies() / stats()."""
        nbytes = dev_gensteps.numel() * dev_gensteps.element_size()
        if not dev_gensteps.is_cuda or not dev_gensteps.is_contiguous() or nbytes % 40:
            raise ValueError("dev_gensteps must be a contiguous CUDA tensor of 40-byte gensteps")
        arr, faces = _events_c(events)
        self._keep = (arr, faces, dev_gensteps)
        _lib.call("optx_engine_set_gensteps_device", self._h, ctypes.cast(arr, ctypes.c_void_p),
                  ctypes.cast(faces, ctypes.c_void_p) if faces is not None else None, len(events),
                  ctypes.c_void_p(dev_gensteps.data_ptr()), nbytes // 40, first_id,
                  ctypes.c_void_p(stream or 0))
        self.n_events = len(events)
        self.counts = None  # known on the device only

    def run_gensteps(self, events, gensteps, first_id: int = 0):
        """One-shot host-buffer genstep run: upload, graph launch, D2H per-event tallies."""
        from .gensteps import as_gensteps
        arr, faces = _events_c(events)
        g = as_gensteps(gensteps)
        out = np.zeros((len(events), self.tally_config.length), np.uint64)
        st = _lib.CEventStats()
        tm = _lib.CTiming()
        _lib.call("optx_run_gensteps", self._h, ctypes.cast(arr, ctypes.c_void_p),
                  ctypes.cast(faces, ctypes.c_void_p) if faces is not None else None, len(events),
                  g.ctypes.data, len(g), first_id, out.ctypes.data, ctypes.byref(st), ctypes.byref(tm))
        self.n_events = len(events)
        return out, st.as_dict(), tm.as_dict()

    def run_tally(self, stream=0):
        _lib.call("optx_engine_run_tally", self._h, ctypes.c_void_p(stream or 0))

    def run_records(self, dev_records, stream=0):
        """Per-photon records of the uploaded batch into device arrays (one entry
        per photon, in batch order). Sizes are checked when the host knows the
        batch's photon count (not after set_gensteps_device)."""
        if self.counts is not None:
            check_records_out(dev_records, int(np.asarray(self.counts, np.uint64).sum()))
        cr = _crec_from_torch(dev_records)
        _lib.call("optx_engine_run_records", self._h, ctypes.byref(cr), ctypes.c_void_p(stream or 0))

    def tallies(self, stream=0) -> np.ndarray:
        """Per-event flat tallies, shape (n_events, tally length)."""
        out = np.zeros((self.n_events, self.tally_config.length), np.uint64)
        _lib.call("optx_engine_get_tallies", self._h, out.ctypes.data, ctypes.c_void_p(stream or 0))
        return out

    def run_tally_range(self, lo: int, hi: int, accumulate: bool = True, stream=0):
        """Transports the batch's relative photons [lo, hi) (photon i of event j
        is offset_j + i) in tally mode, adding to the per-event tallies
        (accumulate=True) or zeroing them first. Consecutive ranges give the
        tallies of one whole run exactly: the unit of checkpoint and resume."""
        _lib.call("optx_engine_run_tally_range", self._h, int(lo), int(hi), 1 if accumulate else 0,
                  ctypes.c_void_p(stream or 0))

    def set_tallies(self, tallies, stream=0):
        """Replaces the per-event tallies (n_events x tally length) with host values."""
        t = np.ascontiguousarray(tallies, dtype=np.uint64)
        if t.shape != (self.n_events, self.tally_config.length):
            raise ValueError(f"tallies must have shape ({self.n_events}, {self.tally_config.length})")
        _lib.call("optx_engine_set_tallies", self._h, t.ctypes.data, ctypes.c_void_p(stream or 0))

    def tally_ptr(self):
        p = ctypes.c_void_p()
        ln = ctypes.c_uint64()
        _lib.call("optx_engine_tally_ptr", self._h, ctypes.byref(p), ctypes.byref(ln))
        return p.value, ln.value

    def stats(self, stream=0) -> dict:
        st = _lib.CEventStats()
        _lib.call("optx_engine_stats", self._h, ctypes.byref(st), ctypes.c_void_p(stream or 0))
        return st.as_dict()

    def run_batch(self, events, counts, first_id: int = 0):
        """One-shot host-buffer run: H2D table, graph launch, D2H tallies."""
        arr, faces = _events_c(events)
        cnt = _counts_c(counts, len(arr))
        out = np.zeros((len(events), self.tally_config.length), np.uint64)
        st = _lib.CEventStats()
        tm = _lib.CTiming()
        _lib.call("optx_run_batch", self._h, ctypes.cast(arr, ctypes.c_void_p),
                  ctypes.cast(faces, ctypes.c_void_p) if faces is not None else None,
                  cnt.ctypes.data, len(events), first_id, out.ctypes.data, ctypes.byref(st),
                  ctypes.byref(tm))
        self.n_events = len(events)
        self.counts = cnt
        return out, st.as_dict(), tm.as_dict()


class SortedEngine:
    """Per-interaction sorted kernels (optx_sorted_*): photons wait between steps
    in state queues sorted by their pending interaction (Rayleigh scatter,
    polished face, painted face); every launch gives each warp 32 photons of one
    kind. Same records as `records_device` bit for bit, same tallies as
    `tally_device`; one configuration per run, asynchronous on the stream."""

    def __init__(self, capacity: int = 0, drain_below: int = 0, math="fast", host_loop: bool = False,
                 blocks_per_sm: int = 0):
        from .backend import _math
        self._h = ctypes.c_void_p()
        cfg = _lib.CSortedConfig(capacity, drain_below, _math(math), blocks_per_sm, 1 if host_loop else 0)
        _lib.call("optx_sorted_create", ctypes.byref(cfg), ctypes.byref(self._h))

    def close(self):
        if self._h:
            _lib.lib().optx_sorted_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, p: SimParams, n: int, first_id: int = 0, tally: TallyConfig | None = None,
            tally_out=None, records_out=None, stream=None, check: bool = False):
        """Runs n photons. With `tally` set, ADDS into `tally_out` (a torch int64
        device tensor of tally.length; a zeroed one is made when None). Records
        go into `records_out` (a dict from backend.device_records) when given.
        Returns (tally_out, records_out).

        The run is asynchronous: a queue overflow or a watchdog stop is reported
        only by the next `stats()` call. With check=True the call synchronises
        the stream and raises on those errors (as `stats()` does)."""
        import torch
        if tally is not None and tally_out is None:
            tally_out = torch.zeros(tally.length, dtype=torch.int64, device="cuda")
        # The kernels write through raw pointers: check sizes and placement here.
        if tally is not None:
            check_tally_out(tally_out, tally.length)
        if records_out is not None:
            check_records_out(records_out, n)
        cp, cf = _lib.params_args(p)
        cc = tally.to_c() if tally is not None else None
        cr = _crec_from_torch(records_out) if records_out is not None else None
        _lib.call("optx_sorted_run", self._h, ctypes.byref(cp), _lib.ref(cf),
                  ctypes.byref(cc) if cc is not None else None, n, first_id,
                  ctypes.c_void_p(tally_out.data_ptr()) if tally is not None else None,
                  ctypes.byref(cr) if cr is not None else None, _stream_ptr(stream))
        if check:
            self.stats(stream)
        return tally_out, records_out

    def stats(self, stream=None) -> dict:
        """Counters of the last run (synchronises the stream)."""
        st = _lib.CSortedCounters()
        _lib.call("optx_sorted_stats", self._h, ctypes.byref(st), _stream_ptr(stream))
        return st.as_dict()


# ---- checkpoint and resume of a batched run ---------------------------------

def batch_fingerprint(events, counts, first_id: int, tally: TallyConfig) -> str:
    """SHA-256 over the batch's C parameter records, photon counts, first id and
    tally binning: a checkpoint resumes only the batch it was taken from."""
    import hashlib
    arr, faces = _events_c(events)
    h = hashlib.sha256()
    h.update(bytes(arr))
    if faces is not None:
        h.update(bytes(faces))
    h.update(np.ascontiguousarray(counts, dtype=np.uint64).tobytes())
    h.update(np.uint64(first_id).tobytes())
    h.update(np.array([tally.time_bins, tally.xy_bins], np.uint32).tobytes())
    h.update(np.float32(tally.time_max).tobytes())
    return h.hexdigest()


def save_checkpoint(path: str, fingerprint: str, next_index: int, tallies) -> None:
    """Writes a checkpoint (.npz format): the batch fingerprint, the next relative
    photon index and the per-event tallies so far. The file is written under
    exactly `path` (no extension is added, so the next run finds it there) and
    replaces the previous checkpoint in one rename: a run killed while writing
    leaves the previous checkpoint intact."""
    import os
    tmp = f"{path}.tmp{os.getpid()}"
    try:
        with open(tmp, "wb") as f:  # a file object: np.savez appends no ".npz"
            np.savez(f, fingerprint=np.array(fingerprint), next_index=np.uint64(next_index),
                     tallies=np.ascontiguousarray(tallies, dtype=np.uint64))
        os.replace(tmp, path)
    finally:
        if os.path.exists(tmp):
            os.remove(tmp)


def load_checkpoint(path: str, fingerprint: str):
    """(next relative photon index, tallies) of a checkpoint taken from the batch
    with this fingerprint; ValueError for another batch."""
    with np.load(path) as z:
        if str(z["fingerprint"]) != fingerprint:
            raise ValueError("the checkpoint was taken from another batch (events, counts, "
                             "first_id or tally binning differ)")
        return int(z["next_index"]), z["tallies"].copy()


def run_tally_checkpointed(engine: "WavefrontEngine", events, counts, first_id: int = 0,
                           path: str | None = None, slice_photons: int = 1 << 24,
                           stop_after: int | None = None):
    """Runs the uploaded batch in slices of `slice_photons` photons, writing a
    checkpoint to `path` after each slice, and resumes from `path` when it
    holds a checkpoint of this batch. `stop_after` ends the call after that
    many slices (an interrupted run). Returns (tallies, next index); the run is
    complete when the next index equals the batch's photon total."""
    import os
    total = int(np.asarray(counts, dtype=np.uint64).sum())
    fp = batch_fingerprint(events, counts, first_id, engine.tally_config)
    start = 0
    if path is not None and os.path.exists(path):
        start, t = load_checkpoint(path, fp)
        engine.set_tallies(t)
    done = 0
    lo = start
    while lo < total and (stop_after is None or done < stop_after):
        hi = min(total, lo + slice_photons)
        engine.run_tally_range(lo, hi, accumulate=lo > 0)
        lo = hi
        done += 1
        if path is not None:
            save_checkpoint(path, fp, lo, engine.tallies())
    if total == 0:
        engine.run_tally()
    return engine.tallies(), lo


def wavefront_tally(p: SimParams, c: TallyConfig, n: int, first_id: int = 0,
                    config: WaveConfig | None = None):
    """Single-configuration tally through the wavefront engine. Returns (Tally, flat, stats)."""
    eng = WavefrontEngine(c, 1, max(n, 1), config)
    try:
        eng.set_events([p], [n], first_id)
        eng.run_tally()
        flat = eng.tallies()[0]
        return Tally.from_flat(flat, c), flat, eng.stats()
    finally:
        eng.close()


# ---- the batched-event workload --------------------------------------------

def batched_events(n_events: int = 4096, seed: int = 2024, median: float = 1e4, sigma: float = 1.0,
                   n_min: int = 100, n_max: int = 1_000_000, photon_seed: int = 12345):
    """Events of the batched configuration (project generator, numpy PCG64 with `seed`).

    Photons per event: lognormal(median, sigma) rounded and clamped to [n_min, n_max].
    Point source uniform in the 50 mm cube; abs_length U(200, 3000) mm; Lambertian
    faces with R U(0.85, 0.99); n_scint U(1.50, 1.70); scat_length inf with p = 0.5,
    else U(300, 1000) mm; n_det = 1.5 and tau = 4 ns (not fixed by the workload
    description, taken from the wrapped-Lambertian setup). All events share the
    Philox key `photon_seed`. Returns (list of SimParams, counts uint64 array).
    """
    rng = np.random.default_rng(seed)
    z = rng.standard_normal(n_events)
    counts = np.clip(np.rint(np.exp(np.log(median) + sigma * z)), n_min, n_max).astype(np.uint64)
    src = rng.uniform(-25.0, 25.0, size=(n_events, 3))
    la = rng.uniform(200.0, 3000.0, n_events)
    refl = rng.uniform(0.85, 0.99, n_events)
    ns = rng.uniform(1.50, 1.70, n_events)
    scat_on = rng.uniform(0.0, 1.0, n_events) >= 0.5
    ls = rng.uniform(300.0, 1000.0, n_events)
    events = []
    for i in range(n_events):
        events.append(SimParams(
            n_scint=float(np.float32(ns[i])), n_det=1.5, abs_length=float(np.float32(la[i])),
            scat_length=float(np.float32(ls[i])) if scat_on[i] else float("inf"),
            surface=LAMBERTIAN, reflectivity=float(np.float32(refl[i])), source=POINT,
            src_x=float(np.float32(src[i, 0])), src_y=float(np.float32(src[i, 1])),
            src_z=float(np.float32(src[i, 2])), tau=4.0, seed=photon_seed))
    return events, counts
