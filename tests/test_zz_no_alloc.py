"""The allocation-free wavefront tally (optx_wavefront_tally_noalloc) against the
history-kernel tally (optx_run_tally): same photons, so the integer tallies must
be equal, on two calls in a row (the static scratch keeps the previous call's
contents and must be cleared by the call itself). Collected last on purpose."""
import ctypes

import numpy as np
import pytest

from gpu_optical_photons_b200 import _lib, params as P

pytestmark = pytest.mark.gpu


def noalloc_tally(p, c, n, first_id=0, math="fast"):
    out = np.full(c.length, 0xDEADBEEF, np.uint64)
    cp, cf = _lib.params_args(p)
    cc = c.to_c()
    L = _lib.lib()
    fn = L.optx_wavefront_tally_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p,
                                           ctypes.c_int, ctypes.c_void_p]
    _lib.check(fn(ctypes.byref(cp), _lib.ref(cf), ctypes.byref(cc), n, first_id,
                  out.ctypes.data, _lib.MATH[math], None))
    return out


@pytest.mark.parametrize("math_mode", ["fast", "exact"])
def test_noalloc_equals_run_tally_twice(engine, math_mode):
    cases = [(P.config2()[0], P.TallyConfig(500, 50.0, 50), 600_000, 3),
             (P.config3(True)[0], P.TallyConfig(100, 20.0, 20), 400_000, 1000)]
    for p, c, n, first_id in cases:
        _, want, _ = engine.run_gpu_tally(p, c, n, first_id=first_id, math=math_mode)
        for _ in range(2):  # the second call must not see the first call's scratch
            got = noalloc_tally(p, c, n, first_id, math_mode)
            assert np.array_equal(got, want)
            assert int(got[:5].sum()) == n


def test_noalloc_rejects_oversized_tally(engine):
    with pytest.raises(ValueError, match="static scratch maximum"):
        noalloc_tally(P.SimParams(), P.TallyConfig(100, 50.0, 300), 1000)
