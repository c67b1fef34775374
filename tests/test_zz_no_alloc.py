"""The allocation-free wavefront tally (optx_wavefront_tally_noalloc).

Some callers cannot call cudaMalloc: code whose device memory belongs to
another runtime's or framework's allocator, or a process that may not grow its
device footprint after start-up. This entry point keeps all of its scratch in a
static array of the library. The array keeps the previous call's contents, so
every case runs two calls in a row: the second must not see the first.

Exact mode must equal the oracle's portable-math tally (the reference's
OPTPHOT_PORTABLE_MATH CPU build, integer tallies, bitwise); fast mode must equal
the cached-engine tally (optx_run_tally), which runs the same photons. The
longest accepted tally is what the opt-in shared memory per block leaves beside
the pantries: a tally of that length runs, one entry more is rejected before any
launch. Collected last on purpose (its name sorts last)."""
import ctypes
import re

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


CASES = [(P.config2()[0], P.TallyConfig(500, 50.0, 50), 600_000, 3),
         (P.config3(True)[0], P.TallyConfig(100, 20.0, 20), 400_000, 1000)]


def test_noalloc_exact_equals_oracle_twice(engine, oracle):
    for p, c, n, first_id in CASES:
        want = oracle.tally(p, c, n, first_id, mode=oracle.PORTABLE)
        for _ in range(2):  # the second call must not see the first call's scratch
            got = noalloc_tally(p, c, n, first_id, "exact")
            assert np.array_equal(got, want)
            assert int(got[:5].sum()) == n


def test_noalloc_fast_equals_run_tally_twice(engine):
    for p, c, n, first_id in CASES:
        _, want, _ = engine.run_gpu_tally(p, c, n, first_id=first_id, math="fast")
        for _ in range(2):
            got = noalloc_tally(p, c, n, first_id, "fast")
            assert np.array_equal(got, want)


def _limit(engine):
    """The device's longest accepted tally, read from the rejection of an
    oversized one (tally length = time_bins + xy_bins^2 + 8)."""
    with pytest.raises(ValueError, match="exceeds the maximum of") as ei:
        noalloc_tally(P.SimParams(), P.TallyConfig(100, 50.0, 300), 1000)
    m = re.search(r"maximum of (\d+) entries", str(ei.value))
    assert m, str(ei.value)
    return int(m.group(1))


def test_noalloc_tally_length_limit(engine, oracle):
    limit = _limit(engine)
    assert 40_000 < limit <= 65_536  # B200: 227 KiB of opt-in shared memory per block
    p = P.config1()[0]
    at = P.TallyConfig(limit - 9, 50.0, 1)  # length = time_bins + 1 + 8 = limit
    assert at.length == limit
    for _ in range(2):
        got = noalloc_tally(p, at, 20_000, 7, "exact")
        assert np.array_equal(got, oracle.tally(p, at, 20_000, 7, mode=oracle.PORTABLE))
    over = P.TallyConfig(limit - 8, 50.0, 1)
    assert over.length == limit + 1
    with pytest.raises(ValueError, match="exceeds the maximum of"):
        noalloc_tally(p, over, 20_000, 7, "exact")
    # A rejected call launches nothing: the next call still gives the right tally.
    p2, c2, n2, f2 = CASES[0]
    assert np.array_equal(noalloc_tally(p2, c2, 50_000, f2, "exact"),
                          oracle.tally(p2, c2, 50_000, f2, mode=oracle.PORTABLE))
