"""Geometry invariants on the oracle's records (the reference's geometry cases,
tests/test_geometry.cpp, checked on whole histories, CPU): every photon ends
inside the closed box; detected photons end on the readout plane z = +hz;
escaped and surface-absorbed photons end on a face; photons absorbed in the
bulk end strictly inside."""
import numpy as np
import pytest

from gpu_optical_photons_b200 import params as P

FATE_DETECTED, FATE_BULK, FATE_SURFACE, FATE_ESCAPED = 0, 1, 2, 3

SETUPS = {
    "polished_cube": P.config1()[0],
    "lambertian_rayleigh_volume": P.config2()[0],
    "long_bar_black_minus_z": P.config3(True)[0],
    "specular_scattering": P.SimParams(surface=P.SPECULAR, reflectivity=0.9, scat_length=400.0),
}


@pytest.mark.parametrize("name", list(SETUPS))
def test_histories_end_on_the_box(oracle, name):
    p = SETUPS[name]
    r = oracle.records(p, 20_000, first_id=11)
    x, y, z = (r[k].astype(np.float64) for k in ("x", "y", "z"))
    h = np.array([p.hx, p.hy, p.hz], np.float32).astype(np.float64)
    assert np.all(np.abs(x) <= h[0]) and np.all(np.abs(y) <= h[1]) and np.all(np.abs(z) <= h[2])
    on_face = (np.abs(x) == h[0]) | (np.abs(y) == h[1]) | (np.abs(z) == h[2])
    det = r["fate"] == FATE_DETECTED
    assert det.any() and np.all(z[det] == h[2])
    ends_on_face = (r["fate"] == FATE_ESCAPED) | (r["fate"] == FATE_SURFACE)
    assert np.all(on_face[ends_on_face])
    bulk = r["fate"] == FATE_BULK
    assert np.all(~on_face[bulk])
    assert np.all(r["path"] >= 0.0) and np.all(r["t"] >= 0.0)
