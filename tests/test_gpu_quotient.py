"""The kernels' hit-map quotient (quot_rn: the rounded reciprocal, a product and
two FMA corrections) equals the IEEE division the reference's binning uses
(transport.hpp:170-181), checked exhaustively on the GPU for every a of several
divisors and on random pairs (tests/cuda/quot_check.cu, built here with nvcc)."""
import os
import subprocess

import pytest

from gpu_optical_photons_b200 import build as B

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def test_reciprocal_fma_quotient_equals_ieee_division(engine, tmp_path):
    exe = str(tmp_path / "quot_check")
    subprocess.run([B.nvcc()] + B.ARCH + ["-O3", "-std=c++17", "-I", B.CSRC, "-I", B.INCLUDE,
                    "-DOPTX_EXACT=0", os.path.join(HERE, "cuda", "quot_check.cu"), "-o", exe],
                   check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.count(" 0 mismatches") == 7, out.stdout
