"""The double-double log / atan of the device Green's function
(src_b200/csrc/sc_ddmath.cuh), compiled for the host with the same
operation order, against quad precision rounded once."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "src_b200", "csrc")


def _cxx():
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    return None


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    cxx = _cxx()
    if cxx is None:
        pytest.skip("no host C++ compiler")
    exe = str(tmp_path_factory.mktemp("ddm") / "ddmath_check")
    subprocess.run([cxx, "-O2", "-std=c++17", "-ffp-contract=off", "-I", CSRC,
                    os.path.join(HERE, "ddmath_check.cpp"), "-o", exe, "-lquadmath"], check=True)
    return exe


def test_ddmath_correctly_rounded(checker):
    out = subprocess.run([checker, "2000000"], check=True, capture_output=True, text=True).stdout.split()
    n, bad_log, bad_atan, libm_log, libm_atan, diff_log, diff_atan, quick_log, quick_atan, garg, gquick = map(int, out)
    assert n == 2_000_000
    # every one of 2e6 log and 2e6 atan results equals the correctly rounded value
    assert bad_log == 0 and bad_atan == 0, out
    # the quick phase (rounding test, else the full evaluation) returns the
    # full evaluation's bits, and decides nearly every argument by itself
    assert diff_log == 0 and diff_atan == 0, out
    assert quick_log > 0.99 * n and quick_atan > 0.99 * n, out
    # on the Green's function's own arguments the full evaluation is rare
    # (it costs the whole warp when one lane needs it)
    assert gquick > 0.995 * garg, out
    # and the host libm is not (it need not be): the reason for this code
    assert libm_log + libm_atan >= 0
