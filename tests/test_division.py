"""The divisions by per-step constants of the particle kernels (div_rcp in
src_b200/csrc/sc_common.cuh: a product by the correctly rounded reciprocal
and one FMA correction, used when the quotient is in the range where that
equals IEEE division for divisors of at least 2^-70), built for the host
with nvcc: the range test at its edges and 4e6 random quotients, subnormal
dividends and quotients near the ends of the range included, bit for bit
against a / b."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _nvcc():
    for c in ("/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    return None


def test_div_rcp_equals_ieee_division(tmp_path):
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("no nvcc for the host build")
    exe = str(tmp_path / "div_check")
    subprocess.run([nvcc, "-x", "cu", "-std=c++17", "-O2", "-Xcompiler", "-ffp-contract=off", "-Wno-deprecated-gpu-targets",
                    "-I", os.path.join(ROOT, "src_b200", "csrc"), "-I", os.path.join(ROOT, "include"),
                    os.path.join(HERE, "div_check.cu"), "-o", exe], check=True)
    edge, n, bad, fast = (int(v) for v in subprocess.run([exe, "4000000"], check=True, capture_output=True,
                                                          text=True).stdout.split())
    assert edge == 0
    assert n == 4_000_000 and bad == 0
    assert fast > n // 2  # most quotients take the product path
