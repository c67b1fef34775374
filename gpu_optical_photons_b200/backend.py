"""Host API of the engine, mirroring the reference's GPU backend.

Same names, argument meaning and error behaviour as include/optphot/backend.hpp
of the reference (zmeskma/GPU_Optical_photons):

=============================  =========================================  ======================
reference (backend.hpp)        here                                        C ABI (include/optx.h)
=============================  =========================================  ======================
gpu_available() :84            gpu_available()                             optx_gpu_available
gpu_device_name() :85          gpu_device_name()                           optx_gpu_device_name
run_gpu_records() :88-89       run_gpu_records(p, n, block_size, ...)      optx_run_records
run_gpu_tally() :90-91         run_gpu_tally(p, c, n, block_size, ...)     optx_run_tally
run_gpu_records_event() :110   run_gpu_records_event(p, n, k, ...)         optx_run_records_event
=============================  =========================================  ======================

Bad block sizes or k = 0 raise ``InvalidArgument`` (a ``ValueError``), as the
reference throws std::invalid_argument (src/gpu/gpu_event.cu:177-182); CUDA
and resource failures raise ``OptxError`` (std::runtime_error there).
``math="exact"`` selects the bit-reproducible build (portable math, no FMA).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from .params import NUM_FATES, SimParams, TallyConfig, DETECTED, ABSORBED_BULK


class Records(dict):
    """Structure-of-arrays photon records (PhotonRecords, backend.hpp:31-50)."""

    FIELDS = ("fate", "n_boundary", "n_scatter", "t", "x", "y", "z", "path")
    BYTES_PER_PHOTON = 29

    DTYPES = {"fate": np.uint8, "n_boundary": np.uint32, "n_scatter": np.uint32, "t": np.float32,
              "x": np.float32, "y": np.float32, "z": np.float32, "path": np.float32}

    @staticmethod
    def empty(n: int) -> "Records":
        r = Records()
        for k in Records.FIELDS:
            r[k] = np.zeros(n, Records.DTYPES[k])
        return r

    def resize(self, n: int) -> "Records":
        """Makes every field a writable, C-contiguous array of n entries of its
        type, replacing the fields that are not (the reference's callee resizes
        the caller's vectors, cpu_backend.cpp:40-49): the C ABI writes n entries
        through each field's pointer."""
        for k in self.FIELDS:
            v = self.get(k)
            if not (isinstance(v, np.ndarray) and v.dtype == self.DTYPES[k] and v.ndim == 1
                    and v.shape[0] == n and v.flags.c_contiguous and v.flags.writeable):
                self[k] = np.zeros(n, self.DTYPES[k])
        return self

    def c_struct(self) -> _lib.CRecords:
        return _lib.CRecords(*[self[k].ctypes.data for k in self.FIELDS])

    def __len__(self):
        return len(self["fate"])

    def steps(self) -> np.ndarray:
        """n_boundary + n_scatter + [absorbed in bulk] (apps/optphot_event_bench.cpp:39-41)."""
        return self["n_boundary"].astype(np.int64) + self["n_scatter"] + (self["fate"] == ABSORBED_BULK)


@dataclass
class Tally:
    """Tally (backend.hpp:52-63) built from the flat u64 layout of the C ABI."""

    fate_counts: np.ndarray
    time_hist: np.ndarray
    xy_hist: np.ndarray
    boundary_sum: int
    scatter_sum: int

    @staticmethod
    def from_flat(flat: np.ndarray, c: TallyConfig) -> "Tally":
        flat = np.asarray(flat, dtype=np.uint64)
        t0 = NUM_FATES
        x0 = t0 + c.time_bins + 1
        s0 = x0 + c.xy_bins * c.xy_bins
        return Tally(flat[:t0].copy(), flat[t0:x0].copy(), flat[x0:s0].copy(),
                     int(flat[s0]), int(flat[s0 + 1]))

    def total(self) -> int:
        return int(self.fate_counts.sum())

    def steps(self) -> int:
        """Photon steps of the run: sum n_boundary + sum n_scatter + absorbed in bulk."""
        return self.boundary_sum + self.scatter_sum + int(self.fate_counts[ABSORBED_BULK])


def gpu_available() -> bool:
    return bool(_lib.lib().optx_gpu_available())


def gpu_device_name() -> str:
    buf = ctypes.create_string_buffer(256)
    _lib.call("optx_gpu_device_name", buf, len(buf))
    return buf.value.decode()


def _math(math) -> int:
    return _lib.MATH[math] if isinstance(math, str) else int(math)


def run_gpu_records(p: SimParams, n: int, block_size: int = 256, first_id: int = 0,
                    chunk: int = 1 << 24, math="fast", out: Records | None = None):
    """Records of photons first_id .. first_id + n - 1 (gpu_backend.cu:119-156). Returns (Records, timing)."""
    out = Records.empty(n) if out is None else out.resize(n)
    cp, cf = _lib.params_args(p)
    cr = out.c_struct()
    tm = _lib.CTiming()
    _lib.call("optx_run_records", ctypes.byref(cp), _lib.ref(cf), n, ctypes.byref(cr), block_size,
              first_id, chunk, _math(math), ctypes.byref(tm))
    return out, tm.as_dict()


def run_gpu_tally(p: SimParams, c: TallyConfig, n: int, block_size: int = 256, first_id: int = 0,
                  math="fast"):
    """Tally of photons first_id .. first_id + n - 1 (gpu_backend.cu:158-212). Returns (Tally, flat, timing)."""
    flat = np.zeros(c.length, np.uint64)
    cp, cf = _lib.params_args(p)
    cc = c.to_c()
    tm = _lib.CTiming()
    _lib.call("optx_run_tally", ctypes.byref(cp), _lib.ref(cf), ctypes.byref(cc), n,
              flat.ctypes.data, block_size, first_id, _math(math), ctypes.byref(tm))
    return Tally.from_flat(flat, c), flat, tm.as_dict()


def run_gpu_records_event(p: SimParams, n: int, steps_per_launch: int, block_size: int = 256,
                          first_id: int = 0, chunk: int = 1 << 24, math="fast"):
    """Wavefront records, bit-identical to run_gpu_records (gpu_event.cu:174-244).

    Returns (Records, EventStats dict, timing)."""
    out = Records.empty(n)
    cp, cf = _lib.params_args(p)
    cr = out.c_struct()
    st = _lib.CEventStats()
    tm = _lib.CTiming()
    _lib.call("optx_run_records_event", ctypes.byref(cp), _lib.ref(cf), n, ctypes.byref(cr),
              steps_per_launch, block_size, first_id, chunk, _math(math), ctypes.byref(st),
              ctypes.byref(tm))
    return out, st.as_dict(), tm.as_dict()


# ---- device-resident calls (torch tensors on cuda) --------------------------

def _stream_ptr(stream):
    if stream is None:
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return ctypes.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else stream)


def device_records(n: int, device="cuda"):
    """A dict of empty torch device arrays for n records."""
    import torch
    d = {"fate": torch.empty(n, dtype=torch.uint8, device=device),
         "n_boundary": torch.empty(n, dtype=torch.int32, device=device),
         "n_scatter": torch.empty(n, dtype=torch.int32, device=device)}
    for k in ("t", "x", "y", "z", "path"):
        d[k] = torch.empty(n, dtype=torch.float32, device=device)
    return d


def check_records_out(d, n: int) -> None:
    """Device record arrays are written through raw pointers: each must be a
    contiguous CUDA tensor of at least n entries of its record field's size."""
    for k in Records.FIELDS:
        v = d[k]
        if not (v.is_cuda and v.is_contiguous() and v.numel() >= n
                and v.element_size() == (1 if k == "fate" else 4)):
            raise ValueError(f"records[{k!r}] must be a contiguous CUDA tensor of >= {n} "
                             f"{'1' if k == 'fate' else '4'}-byte entries")


def check_tally_out(t, length: int) -> None:
    import torch
    if not (t.is_cuda and t.dtype == torch.int64 and t.is_contiguous() and t.numel() >= length):
        raise ValueError(f"tally must be a contiguous int64 CUDA tensor of >= {length} entries")


def _crec_from_torch(d) -> _lib.CRecords:
    return _lib.CRecords(*[d[k].data_ptr() for k in Records.FIELDS])


def records_device(p: SimParams, n: int, first_id: int = 0, out=None, block_size: int = 256,
                   math="fast", stream=None):
    """History kernel into torch device arrays (asynchronous on the stream)."""
    out = device_records(n) if out is None else out
    check_records_out(out, n)
    cp, cf = _lib.params_args(p)
    cr = _crec_from_torch(out)
    _lib.call("optx_records_device", ctypes.byref(cp), _lib.ref(cf), n, first_id, ctypes.byref(cr),
              block_size, _math(math), _stream_ptr(stream))
    return out


def tally_device(p: SimParams, c: TallyConfig, n: int, first_id: int = 0, out=None,
                 block_size: int = 256, math="fast", stream=None, check: bool = True):
    """History tally kernel accumulating into a torch int64 device tensor of
    c.length. `check=False` skips the output check for callers that checked the
    buffer once for many launches."""
    import torch
    out = torch.zeros(c.length, dtype=torch.int64, device="cuda") if out is None else out
    if check:
        check_tally_out(out, c.length)
    cp, cf = _lib.params_args(p)
    cc = c.to_c()
    _lib.call("optx_tally_device", ctypes.byref(cp), _lib.ref(cf), ctypes.byref(cc), n, first_id,
              ctypes.c_void_p(out.data_ptr()), block_size, _math(math), _stream_ptr(stream))
    return out


def records_to_numpy(d) -> Records:
    r = Records()
    for k in Records.FIELDS:
        a = d[k].cpu().numpy()
        if k in ("n_boundary", "n_scatter"):
            a = a.view(np.uint32)
        r[k] = a
    return r
