"""The library divides by its constants (the smoothing weights' sum, the two
convection scales, and in the 3-D field step the neighbour counts 4..7 and
the pressure sweep's 6) with a multiply and two fused multiply-adds instead of a
division (csrc/exact_div.cuh). This checks, for each of those divisors and
every one of the 2^32 f32 inputs, that the result is bit-identical to IEEE
division on the device (tests/cuda/check_exact_div.cu, built here with nvcc
from the library's own header)."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "the-powder-toy-rust-wgpu_b200", "csrc")


def test_division_by_constants_is_exact_for_every_input(cuda, tmp_path):
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    exe = str(tmp_path / "check_exact_div")
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                    "--expt-relaxed-constexpr", "-fmad=false", "-I", CSRC,
                    os.path.join(HERE, "cuda", "check_exact_div.cu"), "-o", exe], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    rows = [line.split() for line in out if line.strip()]
    assert len(rows) == 7
    for divisor, mismatches, first, largest in rows:
        assert int(mismatches) == 0, (divisor, mismatches, first, largest)
