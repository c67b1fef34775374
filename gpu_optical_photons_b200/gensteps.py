"""Gensteps: emission summaries that the engine expands into photons on the GPU.

A genstep (``optx_genstep`` of include/optx.h) describes the photons that one
step of a charged particle emits: a segment (x0,y0,z0)-(x1,y1,z1), an emission
window [t0, t1], a photon count and the event it belongs to. Uploading gensteps
instead of photons is the Opticks approach the reference lists as future work
(README.md section 9 item 7); here the wavefront engine emits each photon when a
warp refills (its position uniform on the segment, its time uniform in the
window plus the event's exponential decay time, its direction isotropic) and
adds it to its event's tally, so no photon list exists anywhere.

``track_gensteps`` cuts a straight track into gensteps with a Poisson photon
yield per step; ``muon_events`` builds a seeded batch of events, each a straight
track crossing the box, as a synthetic genstep workload.
"""
from __future__ import annotations

import numpy as np

from .params import LAMBERTIAN, SimParams

GENSTEP_DTYPE = np.dtype([("x0", "<f4"), ("y0", "<f4"), ("z0", "<f4"), ("t0", "<f4"),
                          ("x1", "<f4"), ("y1", "<f4"), ("z1", "<f4"), ("t1", "<f4"),
                          ("n_photons", "<u4"), ("event", "<u4")])
assert GENSTEP_DTYPE.itemsize == 40

SPEED_OF_LIGHT_MM_NS = 299.792458


def as_gensteps(g) -> np.ndarray:
    """A contiguous GENSTEP_DTYPE array from a structured array, a list of tuples
    in field order or a list of dicts."""
    if isinstance(g, np.ndarray) and g.dtype == GENSTEP_DTYPE:
        return np.ascontiguousarray(g)
    if isinstance(g, np.ndarray) and g.dtype.names:
        out = np.zeros(len(g), GENSTEP_DTYPE)
        for name in GENSTEP_DTYPE.names:
            out[name] = g[name]
        return out
    rows = list(g)
    out = np.zeros(len(rows), GENSTEP_DTYPE)
    for i, r in enumerate(rows):
        if isinstance(r, dict):
            for name in GENSTEP_DTYPE.names:
                out[i][name] = r.get(name, 0)
        else:
            out[i] = tuple(r)
    return out


def to_device(gensteps, device="cuda"):
    """The gensteps as a torch uint8 tensor in device memory (40 bytes per
    genstep, the optx_genstep layout), for WavefrontEngine.set_gensteps_device."""
    import torch
    g = as_gensteps(gensteps)
    return torch.from_numpy(np.ascontiguousarray(g).view(np.uint8)).to(device)


def photons_of(gensteps) -> int:
    return int(np.asarray(as_gensteps(gensteps)["n_photons"], dtype=np.uint64).sum())


def track_gensteps(entry, exit_, photons_per_mm: float, step_mm: float, event: int = 0,
                   t_entry: float = 0.0, beta: float = 1.0, rng=None) -> np.ndarray:
    """Gensteps of a straight track from `entry` to `exit_` (mm) in steps of at
    most `step_mm`; each step emits Poisson(photons_per_mm x step length)
    photons over the time the particle (speed beta c) takes to cross it."""
    rng = rng if rng is not None else np.random.default_rng(0)
    a = np.asarray(entry, np.float64)
    b = np.asarray(exit_, np.float64)
    length = float(np.linalg.norm(b - a))
    n = max(1, int(np.ceil(length / step_mm))) if length > 0 else 1
    f = np.linspace(0.0, 1.0, n + 1)
    pts = a[None, :] + f[:, None] * (b - a)[None, :]
    v = beta * SPEED_OF_LIGHT_MM_NS
    times = t_entry + f * length / v
    seg_len = length / n
    g = np.zeros(n, GENSTEP_DTYPE)
    g["x0"], g["y0"], g["z0"] = pts[:-1, 0], pts[:-1, 1], pts[:-1, 2]
    g["x1"], g["y1"], g["z1"] = pts[1:, 0], pts[1:, 1], pts[1:, 2]
    g["t0"], g["t1"] = times[:-1], times[1:]
    g["n_photons"] = rng.poisson(photons_per_mm * seg_len, n)
    g["event"] = event
    return g


def _box_crossing(rng, h):
    """Entry and exit of a random straight line through the box [-h, h]^3: a
    point uniform in the box and an isotropic direction, extended both ways to
    the faces."""
    p = rng.uniform(-h, h)
    ct = rng.uniform(-1.0, 1.0)
    ph = rng.uniform(0.0, 2 * np.pi)
    st = np.sqrt(1 - ct * ct)
    d = np.array([st * np.cos(ph), st * np.sin(ph), ct])
    with np.errstate(divide="ignore"):
        tpos = np.where(d != 0, (np.sign(d) * h - p) / d, np.inf)
        tneg = np.where(d != 0, (-np.sign(d) * h - p) / d, -np.inf)
    t_out = float(np.min(tpos))
    t_in = float(np.max(tneg))
    return p + t_in * d, p + t_out * d


def muon_events(n_events: int = 256, seed: int = 77, photons_per_mm: float = 200.0,
                step_mm: float = 1.0, size_mm: float = 50.0):
    """A seeded batch of `n_events` events in a `size_mm` cube with Lambertian
    walls (R 0.95, n_det 1.5, scintillation decay 4 ns, absorption and Rayleigh
    lengths 2000 / 500 mm, the physics of the Lambertian validation setup), each
    a straight minimum-ionising track crossing the box, cut into `step_mm`
    gensteps. Returns (events, gensteps)."""
    rng = np.random.default_rng(seed)
    h = np.full(3, size_mm / 2)
    events, parts = [], []
    for e in range(n_events):
        events.append(SimParams(hx=h[0], hy=h[1], hz=h[2], surface=LAMBERTIAN, reflectivity=0.95,
                                n_det=1.5, abs_length=2000.0, scat_length=500.0, tau=4.0,
                                seed=12345))
        a, b = _box_crossing(rng, h)
        parts.append(track_gensteps(a, b, photons_per_mm, step_mm, e, t_entry=0.0, rng=rng))
    return events, np.concatenate(parts)
