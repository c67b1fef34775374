"""Output files in the reference project's layout (src/core/io.cpp, src/core/config.cpp).

A records run writes one NumPy ``.npy`` file per field plus ``meta.json``:

    DIR/fate.npy (|u1)  n_boundary.npy (<u4)  n_scatter.npy (<u4)
        t.npy x.npy y.npy z.npy path.npy (<f4)  meta.json

and a tally run ``fate_counts.npy`` (<u8, 5), ``time_hist.npy`` (<u8,
time_bins + 1) and ``xy_hist.npy`` (<u8, xy_bins x xy_bins) plus ``meta.json``
(io.cpp:48-74), so the reference's Python analysis reads either program's
output. The ``.npy`` writer follows the format's published specification
(version 1.0: magic, header dictionary, spaces and a newline padding the data
offset to a multiple of 64 bytes, little-endian data) and produces the same
bytes as the reference's ``write_npy`` (io.cpp:13-41). ``params_to_json`` gives
the reference's ``meta.json`` text (config.cpp:230-253): the same keys, order,
line breaks and number formatting (floats with 9 significant digits, infinite
lengths as the string "inf").
"""
from __future__ import annotations

import json
import math
import os
import struct
from dataclasses import dataclass, field

import numpy as np

from .backend import Records, Tally
from .params import NUM_FATES, SimParams, TallyConfig

_MAGIC = b"\x93NUMPY\x01\x00"
_DESCR = {np.dtype(np.uint8): "|u1", np.dtype(np.uint32): "<u4", np.dtype(np.float32): "<f4",
          np.dtype(np.uint64): "<u8", np.dtype(np.int64): "<i8", np.dtype(np.float64): "<f8",
          np.dtype(np.int32): "<i4"}
_RECORD_DTYPES = {"fate": np.uint8, "n_boundary": np.uint32, "n_scatter": np.uint32, "t": np.float32,
                  "x": np.float32, "y": np.float32, "z": np.float32, "path": np.float32}
_SURFACES = ["polished", "black", "specular", "lambertian"]
_SOURCES = ["point", "volume"]


def npy_bytes_header(descr: str, shape: tuple) -> bytes:
    """The .npy v1.0 preamble for a C-order array: magic, header length, header."""
    dims = ", ".join(str(int(d)) for d in shape)
    shape_txt = f"({dims},)" if len(shape) == 1 else f"({dims})"
    header = "{'descr': '" + descr + "', 'fortran_order': False, 'shape': " + shape_txt + ", }"
    unpadded = len(_MAGIC) + 2 + len(header) + 1
    header += " " * ((64 - unpadded % 64) % 64) + "\n"
    return _MAGIC + struct.pack("<H", len(header)) + header.encode("latin1")


def write_npy(path: str, array) -> None:
    """Writes `array` (C order, little-endian) as a .npy file."""
    a = np.ascontiguousarray(array)
    if a.dtype.byteorder == ">":
        a = a.astype(a.dtype.newbyteorder("<"))
    descr = _DESCR.get(np.dtype(a.dtype.type))
    if descr is None:
        raise ValueError(f"unsupported dtype {a.dtype}")
    with open(path, "wb") as f:
        f.write(npy_bytes_header(descr, a.shape))
        f.write(a.tobytes(order="C"))


def read_npy(path: str) -> np.ndarray:
    """Reads a .npy file written by `write_npy` or the reference (version 1.0, C order)."""
    with open(path, "rb") as f:
        raw = f.read()
    if raw[:6] != _MAGIC[:6]:
        raise ValueError(f"{path}: not a .npy file")
    major = raw[6]
    if major == 1:
        (hlen,) = struct.unpack("<H", raw[8:10])
        off = 10
    else:
        (hlen,) = struct.unpack("<I", raw[8:12])
        off = 12
    import ast
    hdr = ast.literal_eval(raw[off:off + hlen].decode("latin1"))
    if hdr.get("fortran_order"):
        raise ValueError(f"{path}: Fortran order is not supported")
    dt = np.dtype(hdr["descr"])
    shape = tuple(hdr["shape"])
    count = int(np.prod(shape)) if shape else 1
    data = np.frombuffer(raw, dtype=dt, count=count, offset=off + hlen)
    return data.reshape(shape).copy()


@dataclass
class RunOptions:
    """The run description that meta.json records (config.hpp:19-27)."""

    backend: str = "gpu"
    mode: str = "records"
    n_photons: int = 1_000_000
    threads: int = 1
    block_size: int = 256
    tally: TallyConfig = field(default_factory=TallyConfig)


def _json_float(v: float) -> str:
    f = float(np.float32(v))
    if math.isinf(f):
        return '"inf"'
    return format(f, ".9g")


def params_to_json(p: SimParams, o: RunOptions | None = None) -> str:
    """meta.json text of a run (config.cpp:230-253)."""
    o = o or RunOptions()
    f2 = lambda h: _json_float(np.float32(2) * np.float32(h))  # noqa: E731  (2 * p.hx in float)
    return ("{\n"
            f"  \"size_x\": {f2(p.hx)}, \"size_y\": {f2(p.hy)}, \"size_z\": {f2(p.hz)},\n"
            f"  \"n_scint\": {_json_float(p.n_scint)}, \"n_det\": {_json_float(p.n_det)}, "
            f"\"n_out\": {_json_float(p.n_out)},\n"
            f"  \"abs_length\": {_json_float(p.abs_length)}, \"scat_length\": {_json_float(p.scat_length)},\n"
            f"  \"surface\": \"{_SURFACES[int(p.surface)]}\", \"reflectivity\": {_json_float(p.reflectivity)},\n"
            f"  \"source\": \"{_SOURCES[int(p.source)]}\", \"src_x\": {_json_float(p.src_x)}, "
            f"\"src_y\": {_json_float(p.src_y)}, \"src_z\": {_json_float(p.src_z)},\n"
            f"  \"tau\": {_json_float(p.tau)}, \"max_steps\": {int(p.max_steps)}, \"seed\": {int(p.seed)},\n"
            f"  \"backend\": \"{o.backend}\", \"mode\": \"{o.mode}\", \"n_photons\": {int(o.n_photons)}, "
            f"\"threads\": {int(o.threads)}, \"block_size\": {int(o.block_size)},\n"
            f"  \"time_bins\": {int(o.tally.time_bins)}, \"time_max\": {_json_float(o.tally.time_max)}, "
            f"\"xy_bins\": {int(o.tally.xy_bins)}\n"
            "}")


def write_text_file(path: str, text: str) -> None:
    with open(path, "w") as f:
        f.write(text + "\n")


def write_records(directory: str, rec, meta: str) -> None:
    """DIR/<field>.npy for the eight record fields and DIR/meta.json (io.cpp:48-60)."""
    os.makedirs(directory, exist_ok=True)
    for k, dt in _RECORD_DTYPES.items():
        write_npy(os.path.join(directory, f"{k}.npy"), np.asarray(rec[k]).astype(dt, copy=False))
    write_text_file(os.path.join(directory, "meta.json"), meta)


def write_tally(directory: str, tally: Tally, meta: str) -> None:
    """DIR/fate_counts.npy, time_hist.npy, xy_hist.npy (square) and meta.json (io.cpp:62-72)."""
    os.makedirs(directory, exist_ok=True)
    write_npy(os.path.join(directory, "fate_counts.npy"), np.asarray(tally.fate_counts, dtype=np.uint64))
    write_npy(os.path.join(directory, "time_hist.npy"), np.asarray(tally.time_hist, dtype=np.uint64))
    xy = np.asarray(tally.xy_hist, dtype=np.uint64)
    nb = math.isqrt(xy.size)
    if nb * nb != xy.size:
        raise ValueError(f"xy_hist has {xy.size} entries, not xy_bins x xy_bins")
    write_npy(os.path.join(directory, "xy_hist.npy"), xy.reshape(nb, nb))
    write_text_file(os.path.join(directory, "meta.json"), meta)


def read_records(directory: str) -> Records:
    """Records from a directory written by `write_records` or by the reference."""
    r = Records()
    for k, dt in _RECORD_DTYPES.items():
        a = read_npy(os.path.join(directory, f"{k}.npy"))
        if a.dtype != np.dtype(dt):
            raise ValueError(f"{directory}/{k}.npy: dtype {a.dtype}, expected {np.dtype(dt)}")
        r[k] = a
    return r


def read_tally(directory: str) -> Tally:
    """Tally from a directory written by `write_tally` or by the reference (the two
    step sums are not part of that layout and read as 0)."""
    fc = read_npy(os.path.join(directory, "fate_counts.npy"))
    th = read_npy(os.path.join(directory, "time_hist.npy"))
    xy = read_npy(os.path.join(directory, "xy_hist.npy"))
    if fc.size != NUM_FATES:
        raise ValueError(f"{directory}: fate_counts has {fc.size} entries")
    return Tally(fc, th, xy.reshape(-1), 0, 0)


def read_meta(directory: str) -> dict:
    with open(os.path.join(directory, "meta.json")) as f:
        return json.load(f)
