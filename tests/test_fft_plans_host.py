"""The register-radix FFT plans (16 x 8 ... 16 x 16 x 8, 384 = 16 x 12 x 2)
checked on the host, both as the band kernels run them (band first pass,
middle passes, last pass) and as the row band kernel does (every pass after
the first a middle pass, natural order left in the buffer): csrc/cuda/fft_reg.cuh's pass functions compiled as host
code by nvcc, a 256-thread block emulated thread by thread, against a direct
DFT in double precision (tests/fft_plan_check.cu).  No GPU needed."""
import os
import shutil
import subprocess
import tempfile

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not on PATH")
def test_register_radix_plans_match_direct_dft():
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "fft_plan_check")
        subprocess.run(["nvcc", "-O2", "-std=c++17", "--expt-relaxed-constexpr", "-Wno-deprecated-gpu-targets",
                        "-x", "cu", os.path.join(HERE, "fft_plan_check.cu"), "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    rows = [line.split()[-5:] for line in out.strip().splitlines()]
    assert len(rows) == 29
    for L, S, direction, hb, err in rows:
        # FP32 transforms of unit-scale data: a few ulps of the spectrum's magnitude
        assert float(err) < 1e-6, (L, S, direction, hb, err)
