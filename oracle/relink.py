"""Relinks the reference project's GPU callers against liboptx.so (test infrastructure).

Compiles, from the reference sources where they lie (read only), the programs
that call the reference's GPU backend — its GPU test file tests/test_gpu.cpp and
its apps (apps/optphot_main.cpp, optphot_compare.cpp, optphot_event_bench.cpp,
optphot_bench.cpp) — together with the reference's CPU backend and core
(src/cpu/cpu_backend.cpp, src/core/{compare,config,io}.cpp), and links them with
this repository's C++ shim (gpu_optical_photons_b200/shim/optx_backend.cpp) and
liboptx.so in place of the reference's src/gpu/*.cu. No reference source is
changed or copied; the Catch2 macros of the test file come from
oracle/catch2_min (the reference fetches Catch2 over the network).

Two flavours, as the reference's CMake options give them:

  oracle/_ref/relink/fast/      default build (platform libm; the shim asks for OPTX_MATH_FAST)
  oracle/_ref/relink/portable/  OPTPHOT_PORTABLE_MATH + OPTPHOT_NO_FMAD (the shim asks
                                for OPTX_MATH_EXACT; CPU and GPU histories bitwise identical)

each with gpu_tests, optphot, optphot_compare, optphot_event_bench, optphot_bench.

It also builds the reference's own GPU backend (src/gpu/gpu_backend.cu,
src/gpu/gpu_event.cu) for sm_100a with nvcc, in the same two flavours, behind a
C wrapper (oracle/ref_gpu_capi.cpp): oracle/_ref/libref_gpu.so and
libref_gpu_portable.so, to compare this repository's kernels with the
reference kernels on the same B200.

    python oracle/relink.py [--ref DIR] [--force]

The reference checkout defaults to OPTX_REFERENCE, else to oracle/Makefile's REF.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
from oracle.oracle import reference_root  # noqa: E402  (the checkout: OPTX_REFERENCE or the Makefile's REF)
OUT = os.path.join(HERE, "_ref", "relink")
LIBDIR = os.path.join(ROOT, "gpu_optical_photons_b200")
SHIM = os.path.join(LIBDIR, "shim", "optx_backend.cpp")
CATCH = os.path.join(HERE, "catch2_min")

FLAVOURS = {
    "fast": ["-DOPTPHOT_HAVE_CUDA", "-DOPTPHOT_HAVE_OPENMP"],
    "portable": ["-DOPTPHOT_HAVE_CUDA", "-DOPTPHOT_HAVE_OPENMP", "-DOPTPHOT_PORTABLE_MATH",
                 "-DOPTPHOT_NO_FMAD"],
}
PROGRAMS = {
    "gpu_tests": ["tests/test_gpu.cpp", "@catch_main"],
    "optphot": ["apps/optphot_main.cpp"],
    "optphot_compare": ["apps/optphot_compare.cpp"],
    "optphot_event_bench": ["apps/optphot_event_bench.cpp"],
    "optphot_bench": ["apps/optphot_bench.cpp"],
}
CORE = ["src/cpu/cpu_backend.cpp", "src/core/compare.cpp", "src/core/config.cpp", "src/core/io.cpp"]
CXX = os.environ.get("ORACLE_CXX", "g++")
CXXFLAGS = ["-O3", "-DNDEBUG", "-std=c++17", "-ffp-contract=off", "-fopenmp"]


def _src(ref: str, s: str) -> str:
    if s == "@catch_main":
        return os.path.join(CATCH, "catch_main.cpp")
    if s == "@shim":
        return SHIM
    return os.path.join(ref, s)


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(args):
    src, obj, flags, ref = args
    deps = [src, os.path.join(HERE, "relink.py")]
    if not _stale(obj, deps):
        return
    cmd = [CXX] + CXXFLAGS + flags + ["-I", os.path.join(ref, "include"), "-I",
                                      os.path.join(ROOT, "include"), "-I", CATCH, "-c", src, "-o", obj]
    subprocess.run(cmd, check=True)


NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else "nvcc")
GPU_FLAVOURS = {
    # the reference's CMake: -lineinfo, fmad on by default; OPTPHOT_CUDA_FMAD=OFF -> --fmad=false
    "libref_gpu.so": [],
    "libref_gpu_portable.so": ["-DOPTPHOT_PORTABLE_MATH", "-DOPTPHOT_NO_FMAD", "--fmad=false"],
}


def build_ref_gpu(ref: str | None = None, force: bool = False) -> list[str]:
    """The reference's GPU backend for sm_100a, one shared library per flavour."""
    ref = ref or reference_root()
    if not os.path.isdir(os.path.join(ref, "src", "gpu")):
        return []
    out_dir = os.path.join(HERE, "_ref")
    os.makedirs(out_dir, exist_ok=True)
    srcs = [os.path.join(ref, "src", "gpu", "gpu_backend.cu"), os.path.join(ref, "src", "gpu", "gpu_event.cu"),
            os.path.join(HERE, "ref_gpu_capi.cpp"), os.path.join(ref, "src", "cpu", "cpu_backend.cpp")]
    jobs = []
    for name, flags in GPU_FLAVOURS.items():
        lib = os.path.join(out_dir, name)
        if force or _stale(lib, srcs + [os.path.join(HERE, "relink.py")]):
            jobs.append([NVCC, "-shared", "-O3", "-std=c++17", "-lineinfo",
                         "-gencode", "arch=compute_100a,code=sm_100a",
                         "-Xcompiler", "-fPIC,-ffp-contract=off", "-I", os.path.join(ref, "include")]
                        + flags + srcs + ["-o", lib])
    with ThreadPoolExecutor(max_workers=2) as pool:
        for r in pool.map(lambda c: subprocess.run(c, check=False), jobs):
            if r.returncode != 0:
                raise subprocess.CalledProcessError(r.returncode, r.args)
    return [os.path.join(out_dir, n) for n in GPU_FLAVOURS]


def build(ref: str | None = None, force: bool = False) -> str | None:
    """Builds every program of both flavours; returns the output directory, or
    None when the reference checkout or liboptx.so is missing."""
    ref = ref or reference_root()
    lib = os.path.join(LIBDIR, "liboptx.so")
    if not os.path.isdir(os.path.join(ref, "include", "optphot")) or not os.path.exists(lib):
        return None
    if force and os.path.isdir(OUT):
        shutil.rmtree(OUT)
    jobs, links = [], []
    for fl, flags in FLAVOURS.items():
        d = os.path.join(OUT, fl)
        os.makedirs(d, exist_ok=True)
        objs = {}
        for s in CORE + ["@shim", "@catch_main"] + [p for v in PROGRAMS.values() for p in v if not p.startswith("@")]:
            src = _src(ref, s)
            obj = os.path.join(d, os.path.basename(src).replace(".cpp", ".o"))
            if obj not in objs.values():
                jobs.append((src, obj, flags, ref))
            objs[s] = obj
        for prog, parts in PROGRAMS.items():
            o = [objs[p] for p in parts] + [objs[c] for c in CORE] + [objs["@shim"]]
            links.append((os.path.join(d, prog), o))
    with ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 4)) as pool:
        list(pool.map(_compile, jobs))
    for exe, objs in links:
        if force or _stale(exe, objs + [lib]):
            # rpath: oracle/_ref/relink/<flavour>/ -> the package directory
            cmd = [CXX, "-fopenmp", "-o", exe] + objs + [
                "-L", LIBDIR, "-loptx", "-Wl,-rpath,$ORIGIN/../../../../gpu_optical_photons_b200",
                "-lpthread"]
            subprocess.run(cmd, check=True)
    return OUT


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--ref", default=None, help="reference checkout (default: OPTX_REFERENCE, else the oracle Makefile's REF)")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args(argv)
    build_ref_gpu(a.ref, a.force)
    out = build(a.ref, a.force)
    if out is None:
        print("reference checkout or liboptx.so missing: nothing built", file=sys.stderr)
        return 1
    print(out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
