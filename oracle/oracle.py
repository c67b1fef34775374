"""ctypes wrapper of the CPU oracle (test infrastructure only).

Loads ``oracle/liboptx_oracle.so`` (the project's restatement of the reference
transport, oracle/optx_oracle.cpp) and, when present, ``oracle/_ref/libref_cpu*.so``
(the reference's own CPU backend compiled from its sources by oracle/Makefile).
Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module; the engine in gpu_optical_photons_b200 never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboptx_oracle.so")
REF_SO = {0: os.path.join(HERE, "_ref", "libref_cpu.so"),
          1: os.path.join(HERE, "_ref", "libref_cpu_portable.so")}

PLATFORM, PORTABLE, DOUBLE = 0, 1, 2

_lib = None
_ref = {}

_P = ctypes.c_void_p
_u64 = ctypes.c_uint64


def reference_root() -> str:
    """The reference checkout: the OPTX_REFERENCE environment variable, else the
    default of the build recipe (oracle/Makefile's REF), asked from make."""
    env = os.environ.get("OPTX_REFERENCE")
    if env:
        return env
    r = subprocess.run(["make", "-s", "--no-print-directory", "-C", HERE, "print-ref"],
                       capture_output=True, text=True, check=False)
    return r.stdout.strip() if r.returncode == 0 else ""


def build(with_ref: bool = True) -> None:
    """Builds the oracle (and the reference backend when its checkout is present)."""
    targets = ["all"]
    ref_dir = reference_root()
    if with_ref and ref_dir and os.path.isdir(ref_dir):
        targets.append("ref")
    env = dict(os.environ)
    if ref_dir:
        env["REF"] = ref_dir
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True, env=env)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build(with_ref=False)
        L = ctypes.CDLL(ORACLE_SO)
        L.oracle_records.restype = ctypes.c_int
        L.oracle_records.argtypes = [_P, _P, _u64, _u64, ctypes.c_int, ctypes.c_int] + [_P] * 9
        L.oracle_tally.argtypes = [_P, _P, _P, _u64, _u64, ctypes.c_int, ctypes.c_int, _P]
        L.oracle_batch_tally.argtypes = [_P, _P, ctypes.c_uint32, _P, ctypes.c_int, ctypes.c_int, _P]
        L.oracle_genstep_run.argtypes = [_P, _P, ctypes.c_uint32, _P, _u64, _u64, _P, ctypes.c_int,
                                         ctypes.c_int, _P] + [_P] * 8
        L.oracle_adjoint.argtypes = [_P, _P, _u64, _u64, ctypes.c_int, ctypes.c_int, _P,
                                     ctypes.c_double, _P, _P, _P]
        L.oracle_score_moments.argtypes = [_P, _P, _u64, _u64, ctypes.c_int, ctypes.c_int, _P]
        L.oracle_sample_direction.argtypes = [ctypes.c_int, ctypes.c_float, ctypes.c_float, _P, _P]
        L.oracle_opcount.argtypes = [_P, _P, _u64, _u64, _P]
        L.oracle_stream.argtypes = [_u64, _u64, ctypes.c_uint32, ctypes.c_uint32, _P]
        L.oracle_philox.argtypes = [_P, _P, _P]
        L.oracle_u32_to_uniform.restype = ctypes.c_float
        L.oracle_u32_to_uniform.argtypes = [ctypes.c_uint32]
        L.oracle_portable_log.restype = ctypes.c_float
        L.oracle_portable_log.argtypes = [ctypes.c_float]
        L.oracle_portable_cbrt.restype = ctypes.c_float
        L.oracle_portable_cbrt.argtypes = [ctypes.c_float]
        L.oracle_portable_sincos_turns.argtypes = [ctypes.c_float, _P, _P]
        L.oracle_fresnel.restype = ctypes.c_float
        L.oracle_fresnel.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.c_float]
        L.oracle_rayleigh_cos.restype = ctypes.c_float
        L.oracle_rayleigh_cos.argtypes = [ctypes.c_float, ctypes.c_int]
        _lib = L
    return _lib


def ref_available(mode: int = PLATFORM) -> bool:
    return os.path.exists(REF_SO[mode])


def ref(mode: int = PLATFORM):
    if mode not in _ref:
        L = ctypes.CDLL(REF_SO[mode])
        L.ref_records.restype = ctypes.c_double
        L.ref_records.argtypes = [_P, _u64, _u64, ctypes.c_int] + [_P] * 8
        L.ref_tally.restype = ctypes.c_double
        L.ref_tally.argtypes = [_P, ctypes.c_uint32, ctypes.c_float, ctypes.c_uint32, _u64, _u64,
                                ctypes.c_int, _P]
        L.ref_philox.argtypes = [_P, _P, _P]
        L.ref_max_threads.restype = ctypes.c_int
        L.ref_portable_math.restype = ctypes.c_int
        L.ref_params_to_json.restype = ctypes.c_int
        L.ref_params_to_json.argtypes = [_P, ctypes.c_char_p, ctypes.c_char_p, _u64, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_uint32, ctypes.c_float, ctypes.c_uint32,
                                         ctypes.c_char_p, ctypes.c_size_t]
        L.ref_write_records.restype = ctypes.c_int
        L.ref_write_records.argtypes = [ctypes.c_char_p, _u64] + [_P] * 8 + [ctypes.c_char_p]
        L.ref_write_tally.restype = ctypes.c_int
        L.ref_write_tally.argtypes = [ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint32, _P,
                                      ctypes.c_char_p]
        L.ref_compare_json.restype = ctypes.c_int
        L.ref_compare_json.argtypes = ([_u64] + [_P] * 8 + [_u64] + [_P] * 8 +
                                       [_P, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                        ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t])
        _ref[mode] = L
    return _ref[mode]


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


class Records(dict):
    """Structure-of-arrays photon records (backend.hpp:31-50 field set)."""

    FIELDS = ("fate", "n_boundary", "n_scatter", "t", "x", "y", "z", "path")

    @staticmethod
    def empty(n: int) -> "Records":
        r = Records()
        r["fate"] = np.zeros(n, np.uint8)
        r["n_boundary"] = np.zeros(n, np.uint32)
        r["n_scatter"] = np.zeros(n, np.uint32)
        for k in ("t", "x", "y", "z", "path"):
            r[k] = np.zeros(n, np.float32)
        return r

    def steps(self) -> np.ndarray:
        """Photon steps = n_boundary + n_scatter + [absorbed in bulk] (optphot_event_bench.cpp:39-41)."""
        return (self["n_boundary"].astype(np.int64) + self["n_scatter"]
                + (self["fate"] == 1))


def records(p, n: int, first_id: int = 0, mode: int = PLATFORM, threads: int = 0,
            draws: bool = False) -> Records:
    """Oracle records for photons first_id .. first_id + n - 1."""
    r = Records.empty(n)
    d = np.zeros(n, np.uint32) if draws else None
    cp = p.to_c()
    faces = p.faces_c()
    lib().oracle_records(ctypes.byref(cp), ctypes.byref(faces) if faces is not None else None,
                         n, first_id, mode, threads,
                         *[_ptr(r[k]) for k in Records.FIELDS], _ptr(d))
    if draws:
        r["draws"] = d
    return r


def tally(p, c, n: int, first_id: int = 0, mode: int = PLATFORM, threads: int = 0) -> np.ndarray:
    out = np.zeros(c.length, np.uint64)
    cp, cc = p.to_c(), c.to_c()
    faces = p.faces_c()
    lib().oracle_tally(ctypes.byref(cp), ctypes.byref(faces) if faces is not None else None,
                       ctypes.byref(cc), n, first_id, mode, threads, _ptr(out))
    return out


def batch_tally(events_c, offsets: np.ndarray, c, mode: int = PLATFORM, threads: int = 0,
                n_events: int | None = None) -> np.ndarray:
    """Per-event tallies; events_c is a ctypes array of CSimParams, offsets uint64[n+1]."""
    ne = len(offsets) - 1 if n_events is None else n_events
    out = np.zeros((ne, c.length), np.uint64)
    cc = c.to_c()
    offs = np.ascontiguousarray(offsets, dtype=np.uint64)
    lib().oracle_batch_tally(ctypes.cast(events_c, ctypes.c_void_p), _ptr(offs), ne,
                             ctypes.byref(cc), mode, threads, _ptr(out))
    return out


def genstep_run(events, gensteps, c=None, first_id: int = 0, mode: int = PLATFORM, threads: int = 0,
                records: bool = False):
    """Gensteps (the package's extension): per-event tallies (n_events x len, when
    c is given) and, with records=True, the records of all photons in photon order."""
    from gpu_optical_photons_b200.gensteps import as_gensteps, photons_of
    from gpu_optical_photons_b200.wavefront import _events_c
    arr, faces = _events_c(events)
    g = as_gensteps(gensteps)
    out = None
    cc = None
    if c is not None:
        out = np.zeros((len(events), c.length), np.uint64)
        cc = c.to_c()
    rec = Records.empty(photons_of(g)) if records else None
    ptrs = [_ptr(rec[k]) for k in Records.FIELDS] if records else [None] * 8
    rc = lib().oracle_genstep_run(ctypes.cast(arr, ctypes.c_void_p),
                                  ctypes.cast(faces, ctypes.c_void_p) if faces is not None else None,
                                  len(events), _ptr(g), len(g), first_id,
                                  ctypes.byref(cc) if cc is not None else None, mode, threads,
                                  _ptr(out), *ptrs)
    assert rc == 0
    return out, rec


def adjoint(p, c, n: int, w_bin=None, w_det: float = 0.0, first_id: int = 0,
            mode: int = PLATFORM, threads: int = 0):
    """FP64 score-function gradient sum_photons w * S (see oracle_adjoint)."""
    grad = np.zeros(4, np.float64)
    hist = np.zeros(c.time_bins + 1, np.uint64)
    det = np.zeros(1, np.uint64)
    wb = None if w_bin is None else np.ascontiguousarray(w_bin, np.float64)
    cp, cc = p.to_c(), c.to_c()
    lib().oracle_adjoint(ctypes.byref(cp), ctypes.byref(cc), n, first_id, mode, threads,
                         _ptr(wb), float(w_det), _ptr(grad), _ptr(hist), _ptr(det))
    return grad, hist, int(det[0])


def score_moments(p, c, n: int, first_id: int = 0, mode: int = PLATFORM, threads: int = 0):
    """Per-bin (count, sum of the four scores), shape (time_bins + 1, 5) (see oracle_score_moments)."""
    out = np.zeros((c.time_bins + 1) * 5, np.float64)
    cp, cc = p.to_c(), c.to_c()
    lib().oracle_score_moments(ctypes.byref(cp), ctypes.byref(cc), n, first_id, mode, threads, _ptr(out))
    return out.reshape(-1, 5)


STEP_KINDS = ["start", "absorb", "scatter", "readout_reflect", "detect", "polished_reflect",
              "escape", "black", "painted_absorb", "specular", "lambertian"]


def opcount(p, n: int, first_id: int = 0) -> dict:
    """Algorithmic op counts per step kind: {kind: (steps, fp, transcendental, int)}."""
    out = np.zeros(len(STEP_KINDS) * 4, np.uint64)
    cp = p.to_c()
    faces = p.faces_c()
    lib().oracle_opcount(ctypes.byref(cp), ctypes.byref(faces) if faces is not None else None,
                         n, first_id, _ptr(out))
    out = out.reshape(-1, 4)
    return {k: tuple(int(v) for v in out[i]) for i, k in enumerate(STEP_KINDS)}


def stream(seed: int, photon_id: int, n: int, skip: int = 0) -> np.ndarray:
    out = np.zeros(n, np.uint32)
    lib().oracle_stream(seed, photon_id, skip, n, _ptr(out))
    return out


def philox(ctr, key) -> np.ndarray:
    c = np.ascontiguousarray(ctr, np.uint32)
    k = np.ascontiguousarray(key, np.uint32)
    out = np.zeros(4, np.uint32)
    lib().oracle_philox(_ptr(c), _ptr(k), _ptr(out))
    return out


# ---- the reference's own CPU backend (oracle/_ref) -------------------------

def ref_records(p, n: int, first_id: int = 0, mode: int = PLATFORM, threads: int = 0):
    r = Records.empty(n)
    cp = p.to_c()
    ms = ref(mode).ref_records(ctypes.byref(cp), n, first_id, threads,
                               *[_ptr(r[k]) for k in Records.FIELDS])
    return r, ms


def ref_tally(p, c, n: int, first_id: int = 0, mode: int = PLATFORM, threads: int = 0):
    out = np.zeros(c.length, np.uint64)
    cp = p.to_c()
    ms = ref(mode).ref_tally(ctypes.byref(cp), c.time_bins, c.time_max, c.xy_bins, n, first_id,
                             threads, _ptr(out))
    return out, ms


def ref_philox(ctr, key, mode: int = PLATFORM) -> np.ndarray:
    c = np.ascontiguousarray(ctr, np.uint32)
    k = np.ascontiguousarray(key, np.uint32)
    out = np.zeros(4, np.uint32)
    ref(mode).ref_philox(_ptr(c), _ptr(k), _ptr(out))
    return out


def _rec_ptrs(r):
    arrs = [np.ascontiguousarray(r[k], dtype=dt) for k, dt in
            zip(Records.FIELDS, (np.uint8, np.uint32, np.uint32) + (np.float32,) * 5)]
    return arrs, [_ptr(a) for a in arrs]


def ref_params_to_json(p, backend="gpu", mode="records", n_photons=1_000_000, threads=1,
                       block_size=256, time_bins=100, time_max=50.0, xy_bins=50) -> str:
    """The reference's params_to_json (src/core/config.cpp:230-253)."""
    cp = p.to_c()
    buf = ctypes.create_string_buffer(8192)
    n = ref().ref_params_to_json(ctypes.byref(cp), backend.encode(), mode.encode(), n_photons, threads,
                                 block_size, time_bins, time_max, xy_bins, buf, len(buf))
    assert n >= 0
    return buf.value.decode()


def ref_write_records(directory: str, rec, meta: str) -> None:
    """The reference's write_records (src/core/io.cpp:48-60)."""
    keep, ptrs = _rec_ptrs(rec)
    rc = ref().ref_write_records(directory.encode(), len(keep[0]), *ptrs, meta.encode())
    assert rc == 0


def ref_write_tally(directory: str, c, flat, meta: str) -> None:
    """The reference's write_tally (src/core/io.cpp:62-72)."""
    f = np.ascontiguousarray(flat, dtype=np.uint64)
    assert ref().ref_write_tally(directory.encode(), c.time_bins, c.xy_bins, _ptr(f), meta.encode()) == 0


def ref_compare_json(a, b, p, time_bins=100, t_max=0.0, xy_bins=20):
    """(to_json(compare_histories(a, b)), to_json(compare_distributions(a, b, p, ...)))
    of the reference (src/core/compare.cpp); the first is "null" for different sizes."""
    ka, pa = _rec_ptrs(a)
    kb, pb = _rec_ptrs(b)
    cp = p.to_c()
    h = ctypes.create_string_buffer(4096)
    d = ctypes.create_string_buffer(4096)
    rc = ref().ref_compare_json(len(ka[0]), *pa, len(kb[0]), *pb, ctypes.byref(cp), time_bins, t_max,
                                xy_bins, h, d, len(h))
    assert rc == 0
    return h.value.decode(), d.value.decode()


def compare_histories(a: Records, b: Records) -> dict:
    """Photon-by-photon agreement (reference src/core/compare.cpp:103-127)."""
    discrete = ((a["fate"] == b["fate"]) & (a["n_boundary"] == b["n_boundary"])
                & (a["n_scatter"] == b["n_scatter"]))
    same_bits = discrete.copy()
    for k in ("t", "x", "y", "z", "path"):
        same_bits &= a[k].view(np.uint32) == b[k].view(np.uint32)
    n = len(a["fate"])
    bad = np.nonzero(~discrete)[0]
    return {"n": n, "bitwise_identical": int(same_bits.sum()), "same_discrete": int(discrete.sum()),
            "fate_differs": int((a["fate"] != b["fate"]).sum()),
            "first_divergent": int(bad[0]) if len(bad) else -1}


# ---- the reference's own GPU backend, rebuilt for sm_100a (oracle/_ref) --------

REF_GPU_SO = {PLATFORM: os.path.join(HERE, "_ref", "libref_gpu.so"),
              PORTABLE: os.path.join(HERE, "_ref", "libref_gpu_portable.so")}
_refgpu = {}


def refgpu_available(mode: int = PLATFORM) -> bool:
    return os.path.exists(REF_GPU_SO[mode])


def refgpu(mode: int = PLATFORM):
    if mode not in _refgpu:
        L = ctypes.CDLL(REF_GPU_SO[mode])
        L.refgpu_available.restype = ctypes.c_int
        L.refgpu_records.restype = ctypes.c_int
        L.refgpu_records.argtypes = [_P, _u64, ctypes.c_int, _u64, _u64] + [_P] * 8 + [_P]
        L.refgpu_tally.restype = ctypes.c_int
        L.refgpu_tally.argtypes = [_P, ctypes.c_uint32, ctypes.c_float, ctypes.c_uint32, _u64, ctypes.c_int,
                                   _u64, _P, _P]
        L.refgpu_records_event.restype = ctypes.c_int
        L.refgpu_records_event.argtypes = [_P, _u64, ctypes.c_uint32, ctypes.c_int, _u64, _u64] + [_P] * 8 + [_P, _P]
        _refgpu[mode] = L
    return _refgpu[mode]


def _timing(t):
    return dict(zip(("total_ms", "kernel_ms", "h2d_ms", "d2h_ms", "alloc_ms"), (float(v) for v in t)))


def refgpu_records(p, n: int, first_id: int = 0, mode: int = PLATFORM, block_size: int = 256,
                   chunk: int = 1 << 24):
    """The reference's run_gpu_records (src/gpu/gpu_backend.cu) on this GPU."""
    r = Records.empty(n)
    cp = p.to_c()
    t = np.zeros(5)
    rc = refgpu(mode).refgpu_records(ctypes.byref(cp), n, block_size, first_id, chunk,
                                     *[_ptr(r[k]) for k in Records.FIELDS], _ptr(t))
    assert rc == 0, "reference run_gpu_records threw"
    return r, _timing(t)


def refgpu_tally(p, c, n: int, first_id: int = 0, mode: int = PLATFORM, block_size: int = 256):
    """The reference's run_gpu_tally on this GPU: (flat tally, timing)."""
    out = np.zeros(c.length, np.uint64)
    cp = p.to_c()
    t = np.zeros(5)
    rc = refgpu(mode).refgpu_tally(ctypes.byref(cp), c.time_bins, c.time_max, c.xy_bins, n, block_size,
                                   first_id, _ptr(out), _ptr(t))
    assert rc == 0, "reference run_gpu_tally threw"
    return out, _timing(t)


def refgpu_records_event(p, n: int, k: int, first_id: int = 0, mode: int = PLATFORM, block_size: int = 256,
                         chunk: int = 1 << 24):
    """The reference's run_gpu_records_event (src/gpu/gpu_event.cu) on this GPU."""
    r = Records.empty(n)
    cp = p.to_c()
    st = np.zeros(4)
    t = np.zeros(5)
    rc = refgpu(mode).refgpu_records_event(ctypes.byref(cp), n, k, block_size, first_id, chunk,
                                           *[_ptr(r[k2]) for k2 in Records.FIELDS], _ptr(st), _ptr(t))
    assert rc == 0, "reference run_gpu_records_event threw"
    return r, {"launches": int(st[0]), "useful_lane_steps": int(st[1]), "issued_lane_steps": int(st[2]),
               "kernels_ms": float(st[3])}, _timing(t)
