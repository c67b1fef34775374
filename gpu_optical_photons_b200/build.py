"""Builds liboptx.so in-tree with nvcc for sm_100a.

kernels.cu is compiled three times: with CUDA's math library and FMA
contraction (namespace optx::fast), with the portable math and -fmad=false
(namespace optx::exact), and with --use_fast_math (namespace optx::approx). The CUDA runtime is linked statically so
the library does not depend on the runtime version another module (torch) has
loaded. Run ``python -m gpu_optical_photons_b200.build`` or call ``build()``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liboptx.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", CSRC, "-I", INCLUDE]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps() -> list[str]:
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    files.append(os.path.join(INCLUDE, "optx.h"))
    files.append(os.path.abspath(__file__))
    return files


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles liboptx.so if any source is newer than it; returns its path."""
    deps = _deps()
    if not force and not _stale(LIB, deps):
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    cc = nvcc()
    units = [
        ("kernels_fast.o", "kernels.cu", ["-DOPTX_NS=fast", "-DOPTX_EXACT=0"]),
        ("kernels_exact.o", "kernels.cu", ["-DOPTX_NS=exact", "-DOPTX_EXACT=1", "-fmad=false"]),
        ("kernels_approx.o", "kernels.cu", ["-DOPTX_NS=approx", "-DOPTX_EXACT=0", "--use_fast_math"]),
        ("capi.o", "capi.cu", []),
    ]
    cmds, objs = [], []
    for obj, src, extra in units:
        out = os.path.join(BUILD, obj)
        cmd = [cc] + ARCH + COMMON + extra + ["-c", os.path.join(CSRC, src), "-o", out]
        if verbose:
            cmd += ["-Xptxas", "-v"]
            print(" ".join(cmd), file=sys.stderr)
        cmds.append(cmd)
        objs.append(out)
    with ThreadPoolExecutor(max_workers=len(cmds)) as pool:  # independent units
        for r in pool.map(lambda c: subprocess.run(c, check=False), cmds):
            if r.returncode != 0:
                raise subprocess.CalledProcessError(r.returncode, r.args)
    tmp = LIB + ".tmp"
    cmd = [cc] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs + ["-lpthread", "-ldl", "-lrt"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
