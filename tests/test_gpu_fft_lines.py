"""The register-resident line transforms (passes B, C and D on 64-, 128- and
256-point lines) against the staged shared-memory transforms they replace:
the same Stockham butterflies in the same order, so the same bits.  Each
configuration runs in a fresh process (the kernel choice, SCGPU_FFT_LINES,
is read once per process): open and periodic-z solves, plain and mixed
forms, and one tracked step.
"""
import hashlib
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_SCRIPT = r"""
import hashlib, sys
import numpy as np
sys.path.insert(0, {root!r})
from src_b200 import scgpu
from src_b200.bunch import gaussian_bunch
out = []
rng = np.random.default_rng(3)
for nr in [(32, 32, 32), (64, 64, 64), (128, 128, 128), (32, 64, 128), (64, 128, 32)]:
    rho = np.abs(rng.standard_normal((nr[2], nr[1], nr[0])))
    hr = (2.7e-4, 2.9e-4, 5.1e-3)
    for prec in (scgpu.PLAIN_FP64, scgpu.MIXED):
        with scgpu.Context(nr, precision=prec) as c:
            out.append(hashlib.sha256(c.compute_potential(rho, hr).tobytes()).hexdigest())
            c.set_periodic_z(True)
            out.append(hashlib.sha256(c.compute_potential(rho, hr).tobytes()).hexdigest())
R, P = gaussian_bunch(20000)
with scgpu.Context((64, 64, 64)) as c:
    c.upload(R, P, 1e-12, -1e-9 / 20000, 0.51099892e-03 * 1.0e9)
    c.track(2)
    Rg, Pg = c.download()
    out.append(hashlib.sha256(Rg.tobytes() + Pg.tobytes()).hexdigest())
print("HASHES", " ".join(out))
"""


def _run(lines):
    env = dict(os.environ, SCGPU_FFT_LINES=lines)
    r = subprocess.run([sys.executable, "-c", _SCRIPT.format(root=ROOT)], capture_output=True, text=True, env=env,
                       timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    line = [l for l in r.stdout.splitlines() if l.startswith("HASHES")][0]
    return line.split()[1:]


def test_register_lines_equal_staged_transforms():
    staged, lines = _run("0"), _run("1")
    assert len(staged) == len(lines) == 21
    assert staged == lines
