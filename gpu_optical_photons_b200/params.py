"""Parameter and result structures of the optx C ABI (include/optx.h).

``SimParams`` has the byte layout of the reference's ``optphot::SimParams``
(include/optphot/params.hpp:40-63, 72 bytes) so that the same 72 bytes can be
handed to the reference backend, to this engine's C ABI and to the oracle.
``TallyConfig`` mirrors include/optphot/transport.hpp:164-168 and the enums
mirror include/optphot/params.hpp:61-84.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field, fields

INF = math.inf

# Surface models (params.hpp:61-66).
POLISHED, BLACK, SPECULAR, LAMBERTIAN = 0, 1, 2, 3
SURFACE_NAMES = {"polished": POLISHED, "black": BLACK, "specular": SPECULAR, "lambertian": LAMBERTIAN}
# Sources (params.hpp:68-71).
POINT, VOLUME = 0, 1
# Fates (params.hpp:74-81).
DETECTED, ABSORBED_BULK, ABSORBED_SURFACE, ESCAPED, MAX_STEPS = 0, 1, 2, 3, 4
NUM_FATES = 5
FATE_NAMES = ["detected", "absorbed_bulk", "absorbed_surface", "escaped", "max_steps"]
READOUT_FACE = 5
SPEED_OF_LIGHT = 299.792458  # mm/ns (hd.hpp:37)


class CSimParams(ctypes.Structure):
    """optx_params / optphot::SimParams, 72 bytes."""

    _fields_ = [
        ("hx", ctypes.c_float), ("hy", ctypes.c_float), ("hz", ctypes.c_float),
        ("n_scint", ctypes.c_float), ("n_det", ctypes.c_float), ("n_out", ctypes.c_float),
        ("abs_length", ctypes.c_float), ("scat_length", ctypes.c_float),
        ("surface", ctypes.c_uint32), ("reflectivity", ctypes.c_float),
        ("source", ctypes.c_uint32),
        ("src_x", ctypes.c_float), ("src_y", ctypes.c_float), ("src_z", ctypes.c_float),
        ("tau", ctypes.c_float), ("max_steps", ctypes.c_uint32), ("seed", ctypes.c_uint64),
    ]


assert ctypes.sizeof(CSimParams) == 72


class CFaces(ctypes.Structure):
    """optx_faces: per-face surface model and reflectivity (faces 0..4; 5 is the readout)."""

    _fields_ = [("surface", ctypes.c_uint32 * 6), ("reflectivity", ctypes.c_float * 6)]


class CTallyConfig(ctypes.Structure):
    """optx_tally_config / optphot::TallyConfig."""

    _fields_ = [("time_bins", ctypes.c_uint32), ("time_max", ctypes.c_float), ("xy_bins", ctypes.c_uint32)]


@dataclass
class SimParams:
    """Python view of one simulation setup; defaults are the reference's (params.hpp:40-63)."""

    hx: float = 25.0
    hy: float = 25.0
    hz: float = 25.0
    n_scint: float = 1.63
    n_det: float = 1.63
    n_out: float = 1.0
    abs_length: float = 1000.0
    scat_length: float = INF
    surface: int = POLISHED
    reflectivity: float = 0.95
    source: int = POINT
    src_x: float = 0.0
    src_y: float = 0.0
    src_z: float = 0.0
    tau: float = 4.0
    max_steps: int = 10000
    seed: int = 12345
    # Optional per-face surfaces (faces 0..4); None = `surface` on all five.
    face_surface: list | None = field(default=None)
    face_reflectivity: list | None = field(default=None)

    def to_c(self) -> CSimParams:
        c = CSimParams()
        for f in CSimParams._fields_:
            setattr(c, f[0], getattr(self, f[0]))
        return c

    def faces_c(self) -> CFaces | None:
        if self.face_surface is None and self.face_reflectivity is None:
            return None
        f = CFaces()
        surf = self.face_surface or [self.surface] * 6
        refl = self.face_reflectivity or [self.reflectivity] * 6
        for i in range(6):
            f.surface[i] = int(surf[i]) if i < len(surf) else self.surface
            f.reflectivity[i] = float(refl[i]) if i < len(refl) else self.reflectivity
        return f

    def replace(self, **kw) -> "SimParams":
        d = {f.name: getattr(self, f.name) for f in fields(self)}
        d.update(kw)
        return SimParams(**d)

    @property
    def size(self):
        return (2 * self.hx, 2 * self.hy, 2 * self.hz)


@dataclass
class TallyConfig:
    time_bins: int = 100
    time_max: float = 50.0
    xy_bins: int = 50

    def to_c(self) -> CTallyConfig:
        return CTallyConfig(self.time_bins, self.time_max, self.xy_bins)

    @property
    def length(self) -> int:
        """Flat tally length: [5 fates | time_bins+1 | xy_bins^2 | sum nb | sum ns]."""
        return NUM_FATES + self.time_bins + 1 + self.xy_bins * self.xy_bins + 2


def default_cfg() -> SimParams:
    """configs/default.cfg of the reference: 5 cm cube, polished faces, point source."""
    return SimParams()


def config1() -> tuple[SimParams, TallyConfig]:
    """Plain small: default.cfg with n_det = 1.5; 500 time bins over 0-50 ns, 50x50 hit map."""
    return SimParams(n_det=1.5), TallyConfig(time_bins=500, time_max=50.0, xy_bins=50)


def config2() -> tuple[SimParams, TallyConfig]:
    """Wrapped Lambertian with Rayleigh scattering, volume source."""
    p = SimParams(surface=LAMBERTIAN, reflectivity=0.95, n_det=1.5, abs_length=2000.0,
                  scat_length=500.0, source=VOLUME, tau=4.0)
    return p, TallyConfig(time_bins=500, time_max=50.0, xy_bins=50)


def config3(black_minus_z: bool = True) -> tuple[SimParams, TallyConfig]:
    """Long bar 10x10x200 mm: four specular sides R=0.98, -z black (per-face), point source at z=-80."""
    p = SimParams(hx=5.0, hy=5.0, hz=100.0, surface=SPECULAR, reflectivity=0.98, n_det=1.5,
                  n_scint=1.58, abs_length=3000.0, scat_length=INF, src_z=-80.0, tau=2.1)
    if black_minus_z:
        p.face_surface = [SPECULAR, SPECULAR, SPECULAR, SPECULAR, BLACK, SPECULAR]
        p.face_reflectivity = [0.98] * 6
    return p, TallyConfig(time_bins=500, time_max=50.0, xy_bins=50)


def black_box() -> SimParams:
    """Analytic-test setup (tests/test_transport_cpu.cpp:41-49 of the reference)."""
    return SimParams(surface=BLACK, n_det=1.63, abs_length=INF, scat_length=INF, tau=0.0)
