"""EventTable: the C layout of a batch built once equals the per-call conversion,
with and without per-face surfaces (CPU only)."""
import ctypes

from gpu_optical_photons_b200 import params as P
from gpu_optical_photons_b200.wavefront import EventTable, _events_c, batched_events


def test_event_table_equals_per_call_conversion():
    events, _ = batched_events(n_events=64)
    tab = EventTable(events)
    arr, faces = _events_c(events)
    assert len(tab) == 64 and faces is None and tab.faces is None
    assert bytes(tab.arr) == bytes(arr)
    assert _events_c(tab) == (tab.arr, tab.faces)


def test_event_table_with_per_face_surfaces():
    mixed = P.SimParams(face_surface=[P.LAMBERTIAN, P.POLISHED, P.SPECULAR, P.BLACK, P.LAMBERTIAN, 0],
                        face_reflectivity=[0.9, 0.95, 0.97, 0.5, 0.85, 0.0])
    events = [P.config2()[0], mixed, P.config1()[0]]
    tab = EventTable(events)
    arr, faces = _events_c(events)
    assert faces is not None and bytes(tab.faces) == bytes(faces) and bytes(tab.arr) == bytes(arr)
    assert ctypes.sizeof(tab.faces) == 3 * 48


def test_counts_must_match_the_events():
    """The engine calls read one photon count per event through a raw pointer:
    counts of another length (or shape) are refused before the call."""
    import numpy as np
    import pytest
    from gpu_optical_photons_b200.wavefront import _counts_c
    assert _counts_c([3, 4, 5], 3).dtype == np.uint64
    for bad in ([3, 4], [3, 4, 5, 6], [[3, 4, 5]]):
        with pytest.raises(ValueError, match="one photon count per event"):
            _counts_c(bad, 3)
