"""ctypes binding of liboptx.so (the C ABI declared in include/optx.h).

The library is built in-tree (gpu_optical_photons_b200/liboptx.so) by
``gpu_optical_photons_b200.build``. There is no fallback: if the library is
missing or no GPU is present, the calls raise.
"""
from __future__ import annotations

import ctypes
import os

from .params import CSimParams, CFaces, CTallyConfig

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboptx.so")

OK = 0
ERR_NAMES = {1: "invalid argument", 2: "runtime error", 3: "CUDA error", 4: "no device",
             5: "queue capacity", 6: "watchdog"}
MATH = {"fast": 0, "exact": 1, "approx": 2}


class OptxError(RuntimeError):
    """A non-zero status from liboptx; `code` is the OPTX_ERR_* value."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"optx {ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


class InvalidArgument(OptxError, ValueError):
    """OPTX_ERR_INVALID_ARGUMENT (the reference's std::invalid_argument)."""


class CRecords(ctypes.Structure):
    _fields_ = [("fate", ctypes.c_void_p), ("n_boundary", ctypes.c_void_p),
                ("n_scatter", ctypes.c_void_p), ("t", ctypes.c_void_p), ("x", ctypes.c_void_p),
                ("y", ctypes.c_void_p), ("z", ctypes.c_void_p), ("path", ctypes.c_void_p)]


class CTiming(ctypes.Structure):
    _fields_ = [("total_ms", ctypes.c_double), ("kernel_ms", ctypes.c_double),
                ("h2d_ms", ctypes.c_double), ("d2h_ms", ctypes.c_double),
                ("alloc_ms", ctypes.c_double)]

    def as_dict(self):
        return {f[0]: getattr(self, f[0]) for f in self._fields_}


class CEventStats(ctypes.Structure):
    _fields_ = [("launches", ctypes.c_uint64), ("useful_lane_steps", ctypes.c_uint64),
                ("issued_lane_steps", ctypes.c_uint64), ("kernels_ms", ctypes.c_double),
                ("spills", ctypes.c_uint64)]

    def as_dict(self):
        d = {f[0]: getattr(self, f[0]) for f in self._fields_}
        d["simt_efficiency"] = (self.useful_lane_steps / self.issued_lane_steps
                                if self.issued_lane_steps else 0.0)
        return d


class CSortedConfig(ctypes.Structure):
    _fields_ = [("capacity", ctypes.c_uint32), ("drain_below", ctypes.c_uint32), ("math", ctypes.c_int32),
                ("blocks_per_sm", ctypes.c_int32), ("host_loop", ctypes.c_uint32)]


class CSortedCounters(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_uint64), ("queued", ctypes.c_uint64 * 3),
                ("drained", ctypes.c_uint64), ("kernel_ms", ctypes.c_double)]

    def as_dict(self):
        return {"iterations": self.iterations,
                "queued": dict(zip(("scatter", "polished", "painted"), list(self.queued))),
                "drained": self.drained, "kernel_ms": self.kernel_ms}


class CWaveConfig(ctypes.Structure):
    _fields_ = [("block_size", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32),
                ("threshold", ctypes.c_uint32), ("cadence", ctypes.c_uint32),
                ("wave_quota", ctypes.c_uint64), ("use_graph", ctypes.c_int32),
                ("math", ctypes.c_int32), ("chunk", ctypes.c_uint32),
                ("max_gensteps", ctypes.c_uint32), ("tail_steps", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32)]


class CGenstep(ctypes.Structure):
    """optx_genstep: 40 bytes."""
    _fields_ = [("x0", ctypes.c_float), ("y0", ctypes.c_float), ("z0", ctypes.c_float),
                ("t0", ctypes.c_float), ("x1", ctypes.c_float), ("y1", ctypes.c_float),
                ("z1", ctypes.c_float), ("t1", ctypes.c_float), ("n_photons", ctypes.c_uint32),
                ("event", ctypes.c_uint32)]


_P = ctypes.c_void_p
_u64 = ctypes.c_uint64
_int = ctypes.c_int
_lib = None

# name -> argtypes (restype int unless noted)
_SIGS = {
    "optx_abi_version": [],
    "optx_gpu_available": [],
    "optx_gpu_device_name": [ctypes.c_char_p, ctypes.c_size_t],
    "optx_release_cache": [],
    "optx_run_records": [_P, _P, _u64, _P, _int, _u64, _u64, _int, _P],
    "optx_run_tally": [_P, _P, _P, _u64, _P, _int, _u64, _int, _P],
    "optx_run_records_event": [_P, _P, _u64, _P, ctypes.c_uint32, _int, _u64, _u64, _int, _P, _P],
    "optx_records_device": [_P, _P, _u64, _u64, _P, _int, _int, _P],
    "optx_tally_device": [_P, _P, _P, _u64, _u64, _P, _int, _int, _P],
    "optx_engine_create": [_P, ctypes.c_uint32, _u64, _P, _P],
    "optx_engine_destroy": [_P],
    "optx_engine_set_events": [_P, _P, _P, _P, ctypes.c_uint32, _u64, _P],
    "optx_engine_run_tally": [_P, _P],
    "optx_engine_run_tally_range": [_P, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, _P],
    "optx_engine_set_tallies": [_P, _P, _P],
    "optx_engine_run_records": [_P, _P, _P],
    "optx_engine_run_adjoint": [_P, _P, ctypes.c_double, _P, _P],
    "optx_engine_run_score_moments": [_P, _P, _P],
    "optx_wavefront_tally_noalloc": [_P, _P, _P, _u64, _u64, _P, _int, _P],
    "optx_sorted_create": [_P, _P],
    "optx_sorted_destroy": [_P],
    "optx_sorted_run": [_P, _P, _P, _P, _u64, _u64, _P, _P, _P],
    "optx_sorted_stats": [_P, _P, _P],
    "optx_engine_tally_ptr": [_P, _P, _P],
    "optx_engine_get_tallies": [_P, _P, _P],
    "optx_engine_stats": [_P, _P, _P],
    "optx_run_batch": [_P, _P, _P, _P, ctypes.c_uint32, _u64, _P, _P, _P],
    "optx_engine_set_gensteps": [_P, _P, _P, ctypes.c_uint32, _P, ctypes.c_uint32, _u64, _P],
    "optx_engine_set_gensteps_device": [_P, _P, _P, ctypes.c_uint32, _P, ctypes.c_uint32, _u64, _P],
    "optx_run_gensteps": [_P, _P, _P, ctypes.c_uint32, _P, ctypes.c_uint32, _u64, _P, _P, _P],
}


def lib():
    """Loads liboptx.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OptxError(2, f"{LIB_PATH} is missing: run `python -m gpu_optical_photons_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        L.optx_last_error.restype = ctypes.c_char_p
        L.optx_last_error.argtypes = []
        _lib = L
    return _lib


def declared_symbols() -> list[str]:
    """Every function name this binding expects the library to export."""
    return sorted(list(_SIGS) + ["optx_last_error"])


def check(rc: int) -> None:
    if rc != OK:
        msg = lib().optx_last_error().decode(errors="replace")
        if rc == 1:
            raise InvalidArgument(rc, msg)
        raise OptxError(rc, msg)


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))


def ref(obj):
    return ctypes.byref(obj) if obj is not None else None


def params_args(p):
    """(byref(CSimParams), byref(CFaces) or None) for a SimParams, keeping the structs alive."""
    cp = p.to_c() if not isinstance(p, CSimParams) else p
    cf = p.faces_c() if not isinstance(p, CSimParams) else None
    return cp, cf
