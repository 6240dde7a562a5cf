"""GPU test of scgpu_compute_potential_noalloc, the Poisson solve for callers
that cannot allocate device memory (their device memory belongs to their own
pool allocator, or cudaMalloc's device synchronisation is too costly in their
loop).  The entry point works only on buffers the caller hands it plus fixed
arrays inside the library.

Its results must equal the allocating entry point scgpu_compute_potential's
bit for bit on the same input (same kernels, same twiddle values), over two
calls in a row (the second call finds the first call's data in the shared
scratch).  One test runs in a fresh process whose first library call is the
no-allocation solve, as a host that never creates a context uses it.  This
file is collected last so that a run stopping at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOL_ORACLE = 1e-12  # device vs the CPU oracle (FFT rounding)


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _entry(gpu):
    f = gpu.lib().scgpu_compute_potential_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double), C.c_void_p]
    f.restype = C.c_int
    return f


def test_noalloc_matches_allocating_entry_point(gpu):
    import torch

    f = _entry(gpu)
    rng = np.random.default_rng(7)
    cases = [((32, 24, 16), (2.7e-4, 3.1e-4, 4.9e-3)), ((16, 32, 24), (1.0e-3, 0.8e-3, 2.0e-3))]
    inputs, expected = [], []
    for nr, hr in cases:
        rho = rng.random((nr[2], nr[1], nr[0]))
        with gpu.Context(nr) as c:
            expected.append(c.compute_potential(rho, hr))
        inputs.append(rho)
    stream = torch.cuda.current_stream()
    outs = []
    for (nr, hr), rho in zip(cases, inputs):  # two calls in a row
        d_rho = torch.from_numpy(rho).cuda()
        d_phi = torch.empty_like(d_rho)
        rc = f(d_rho.data_ptr(), d_phi.data_ptr(), nr[0], nr[1], nr[2], (C.c_double * 3)(*hr), stream.cuda_stream)
        assert rc == 0
        outs.append(d_phi)
    torch.cuda.synchronize()
    for out, exp in zip(outs, expected):
        np.testing.assert_array_equal(out.cpu().numpy(), exp)


def test_noalloc_in_place_and_limits(gpu):
    import torch

    f = _entry(gpu)
    rng = np.random.default_rng(8)
    nr, hr = (24, 24, 32), (5e-4, 5e-4, 5e-4)
    rho = rng.random((nr[2], nr[1], nr[0]))
    with gpu.Context(nr) as c:
        exp = c.compute_potential(rho, hr)
    d = torch.from_numpy(rho).cuda()
    assert f(d.data_ptr(), d.data_ptr(), nr[0], nr[1], nr[2], (C.c_double * 3)(*hr), None) == 0
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d.cpu().numpy(), exp)
    # beyond the static scratch: a clear error, nothing enqueued
    big = torch.zeros(33 * 32 * 32, dtype=torch.float64, device="cuda")
    assert f(big.data_ptr(), big.data_ptr(), 33, 32, 32, (C.c_double * 3)(*hr), None) == -8
    assert f(big.data_ptr(), big.data_ptr(), 7, 8, 8, (C.c_double * 3)(*hr), None) == -8
    assert f(None, big.data_ptr(), 8, 8, 8, (C.c_double * 3)(*hr), None) == -1
    assert f(big.data_ptr(), big.data_ptr(), 8, 8, 8, (C.c_double * 3)(5e-4, float("inf"), 5e-4), None) == -1


def test_noalloc_rejects_host_and_short_buffers(gpu):
    """Pointers the GPU must not be handed are refused before any launch:
    host memory, and a device allocation smaller than the mesh (as far as
    the driver reports allocation extents: a block that a pool allocator
    carved out of a larger allocation is checked against that allocation)."""
    import torch

    f = _entry(gpu)
    nr, hr = (16, 16, 16), (1e-3, 1e-3, 1e-3)
    from device_buffers import short_device_buffer

    host = np.zeros(16 ** 3)
    dev = torch.zeros(16 ** 3, dtype=torch.float64, device="cuda")
    h = (C.c_double * 3)(*hr)
    assert f(host.ctypes.data, dev.data_ptr(), *nr, h, None) == -1
    assert f(dev.data_ptr(), host.ctypes.data, *nr, h, None) == -1
    with short_device_buffer(8 * (16 ** 3 // 2)) as short:
        if short is not None:
            assert f(short, dev.data_ptr(), *nr, h, None) == -1
    # the buffers were left alone and the library still works
    torch.cuda.synchronize()
    assert f(dev.data_ptr(), dev.data_ptr(), *nr, h, None) == 0
    torch.cuda.synchronize()


_FRESH = r"""
import ctypes as C, sys
import numpy as np, torch
sys.path.insert(0, {root!r})
from src_b200 import scgpu
from oracle import oracle as O
f = scgpu.lib().scgpu_compute_potential_noalloc
f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double), C.c_void_p]
f.restype = C.c_int
rng = np.random.default_rng(11)
nr, hr = (24, 16, 32), (4e-4, 6e-4, 3e-3)
rho = rng.random((nr[2], nr[1], nr[0]))
d_rho = torch.from_numpy(rho).cuda()
outs = []
for _ in range(2):  # the library's first call, then a second on the same scratch
    d_phi = torch.empty_like(d_rho)
    assert f(d_rho.data_ptr(), d_phi.data_ptr(), *nr, (C.c_double * 3)(*hr), None) == 0
    outs.append(d_phi)
torch.cuda.synchronize()
a, b = (o.cpu().numpy() for o in outs)
assert np.array_equal(a, b)
O.lib(); O.use_reference_fft(False)
ref = O.compute_potential(rho, hr)
err = float(np.max(np.abs(a - ref)) / np.max(np.abs(ref)))
assert err < {tol}, err
with scgpu.Context(nr) as c:  # a context made after it computes the same bits
    assert np.array_equal(c.compute_potential(rho, hr), a)
print("fresh ok", err)
"""


def test_noalloc_first_call_in_fresh_process(gpu):
    """A host that never creates a context: the no-allocation solve is the
    process's first library call (its device set-up runs there)."""
    code = _FRESH.format(root=ROOT, tol=TOL_ORACLE)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "fresh ok" in r.stdout
