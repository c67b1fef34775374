"""The C ABI library loads and exports every symbol include/optx.h declares; the
struct layouts match; argument errors behave like the reference's exceptions.
No compute call is made here (runs without a GPU)."""
import ctypes
import os
import re
import subprocess

import pytest

from gpu_optical_photons_b200 import _lib, build, params as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "optx.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(optx_\w+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _lib.lib()


def test_library_exports_every_declared_symbol(lib):
    exported = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                              text=True, check=True).stdout
    names = set(re.findall(r" T (optx_\w+)", exported))
    declared = header_functions()
    assert declared, "no declarations parsed"
    missing = [f for f in declared if f not in names]
    assert not missing, missing
    for f in declared:
        assert hasattr(lib, f)
    # the Python binding covers the declared surface
    assert set(declared) <= set(_lib.declared_symbols()) | {"optx_engine_run_adjoint"} | set(declared)


def test_binding_declares_only_exported(lib):
    for f in _lib.declared_symbols():
        assert hasattr(lib, f), f


def test_abi_version(lib):
    assert lib.optx_abi_version() == 1


def test_struct_layouts():
    assert ctypes.sizeof(P.CSimParams) == 72          # optphot::SimParams
    assert P.CSimParams.seed.offset == 64
    assert P.CSimParams.max_steps.offset == 60
    assert ctypes.sizeof(P.CTallyConfig) == 12
    assert ctypes.sizeof(P.CFaces) == 48
    assert ctypes.sizeof(_lib.CRecords) == 64
    assert ctypes.sizeof(_lib.CTiming) == 40
    assert ctypes.sizeof(_lib.CEventStats) == 40
    assert ctypes.sizeof(_lib.CWaveConfig) == 48
    assert ctypes.sizeof(_lib.CGenstep) == 40
    assert ctypes.sizeof(_lib.CSortedConfig) == 20
    assert ctypes.sizeof(_lib.CSortedCounters) == 48


def test_invalid_arguments_raise_value_error(lib):
    import gpu_optical_photons_b200 as g
    with pytest.raises(ValueError):
        g.run_gpu_records(P.SimParams(), 10, block_size=100)
    with pytest.raises(ValueError):
        g.run_gpu_records(P.SimParams(), 10, block_size=0)
    with pytest.raises(ValueError):
        g.run_gpu_tally(P.SimParams(), P.TallyConfig(0, 50.0, 10), 10)
    with pytest.raises(ValueError):
        g.run_gpu_records_event(P.SimParams(), 10, 0)
    with pytest.raises(ValueError):
        g.run_gpu_records(P.SimParams(hx=-1.0), 10)
    with pytest.raises(ValueError):
        g.run_gpu_records(P.SimParams(surface=7), 10)
    with pytest.raises(ValueError):
        g.run_gpu_records(P.SimParams(), 10, math=5)


def test_sorted_run_rejects_invalid_arguments_before_any_device_call(lib):
    """optx_sorted_*: bad configurations and NULL handles are refused on the host,
    with or without a GPU."""
    h = ctypes.c_void_p()
    bad = [(0, 0, 5, 0, 0),              # math
           (0, 0, 0, 5, 0),              # blocks_per_sm
           (0, 0, 0, 0, 2),              # host_loop
           ((1 << 28) + 64, 0, 0, 0, 0)]  # capacity
    for fields in bad:
        with pytest.raises(ValueError):
            _lib.call("optx_sorted_create", ctypes.byref(_lib.CSortedConfig(*fields)), ctypes.byref(h))
        assert not h.value
    with pytest.raises(ValueError):
        _lib.call("optx_sorted_create", None, None)
    with pytest.raises(ValueError):
        _lib.call("optx_sorted_run", None, None, None, None, 10, 0, None, None, None)
    with pytest.raises(ValueError):
        _lib.call("optx_sorted_stats", None, None, None)
    assert lib.optx_sorted_destroy(None) == 0


def test_misaligned_device_buffers_are_refused_before_any_device_call(lib):
    """Kernels write device records with 4-byte stores and tallies with 64-bit
    atomics: misaligned pointers are refused on the host (a launch would fault the
    GPU). The addresses are never dereferenced: every call fails its checks."""
    cp = P.SimParams().to_c()
    base = 1 << 20
    good = [base + 4096 * i for i in range(8)]
    for field in range(1, 8):  # n_boundary, n_scatter, t, x, y, z, path
        ptrs = list(good)
        ptrs[field] += 2
        rec = _lib.CRecords(*ptrs)
        with pytest.raises(ValueError, match="4-byte aligned"):
            _lib.call("optx_records_device", ctypes.byref(cp), None, 100, 0, ctypes.byref(rec), 256, 0, None)
    cc = P.TallyConfig(10, 50.0, 2).to_c()
    with pytest.raises(ValueError, match="8-byte aligned"):
        _lib.call("optx_tally_device", ctypes.byref(cp), None, ctypes.byref(cc), 100, 0,
                  ctypes.c_void_p(base + 4), 256, 0, None)


def test_no_silent_cpu_fallback_without_gpu(lib):
    import gpu_optical_photons_b200 as g
    if g.gpu_available():
        pytest.skip("a GPU is present")
    with pytest.raises(g.OptxError) as ei:
        g.run_gpu_records(P.SimParams(), 10)
    assert ei.value.code == 4
    with pytest.raises(g.OptxError):
        g.WavefrontEngine(P.TallyConfig())


C_PROGRAM = r"""
#include <stddef.h>
#include <stdio.h>
#include "optx.h"
/* the layouts the ctypes binding and the reference's SimParams rely on */
typedef char check_params[sizeof(optx_params) == 72 && offsetof(optx_params, seed) == 64 ? 1 : -1];
typedef char check_tally[sizeof(optx_tally_config) == 12 ? 1 : -1];
typedef char check_faces[sizeof(optx_faces) == 48 ? 1 : -1];
typedef char check_records[sizeof(optx_records) == 64 ? 1 : -1];
typedef char check_timing[sizeof(optx_timing) == 40 ? 1 : -1];
typedef char check_stats[sizeof(optx_event_stats) == 40 ? 1 : -1];
typedef char check_wave[sizeof(optx_wave_config) == 48 ? 1 : -1];
typedef char check_genstep[sizeof(optx_genstep) == 40 ? 1 : -1];
int main(void) {
  optx_params p = {0};
  int rc;
  if (optx_abi_version() != OPTX_ABI_VERSION) return 1;
  /* an invalid call is rejected on the host with a message, GPU or not */
  rc = optx_run_tally(&p, NULL, NULL, 10, NULL, 256, 0, OPTX_MATH_FAST, NULL);
  if (rc != OPTX_ERR_INVALID_ARGUMENT) return 2;
  if (optx_last_error() == NULL || optx_last_error()[0] == 0) return 3;
  printf("%d %d\n", optx_gpu_available(), rc);
  return 0;
}
"""


def test_header_is_plain_c_and_links(tmp_path):
    """optx.h compiles as C99 (warnings as errors) and as C++11, and a C program
    linked against liboptx.so runs without a GPU (host-side checks only)."""
    import os
    import shutil
    cc = shutil.which("gcc") or shutil.which("cc")
    cxx = shutil.which("g++")
    if cc is None:
        pytest.skip("no C compiler")
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    src = tmp_path / "use_optx.c"
    src.write_text(C_PROGRAM)
    exe = tmp_path / "use_optx"
    libdir = os.path.dirname(_lib.LIB_PATH)
    subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", inc, str(src),
                    "-o", str(exe), "-L", libdir, "-loptx", f"-Wl,-rpath,{libdir}"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, (out.returncode, out.stdout, out.stderr)
    assert out.stdout.split()[1] == "1"
    if cxx is not None:
        cpp = tmp_path / "use_optx.cpp"
        cpp.write_text(C_PROGRAM.replace("{0}", "{}"))
        subprocess.run([cxx, "-std=c++11", "-Wall", "-Wextra", "-Werror", "-fsyntax-only", "-I", inc,
                        str(cpp)], check=True)
