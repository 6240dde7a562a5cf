"""GPU test of scgpu_compute_potential_noalloc, the Poisson solve for callers
that cannot allocate device memory (their device memory belongs to their own
pool allocator, or cudaMalloc's device synchronisation is too costly in their
loop).  The entry point works only on buffers the caller hands it plus a
fixed scratch array inside the library.

Its results must match the allocating entry point scgpu_compute_potential on
the same input, over two calls in a row (the second call finds the first
call's data in the shared scratch).  This file is collected last so that a
run stopping at the first failure has already run every other test; it also
passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12  # device vs device: only the twiddle factors are computed differently


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
        assert rel(out.cpu().numpy(), exp) < TOL


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
    assert rel(d.cpu().numpy(), exp) < TOL
    # beyond the static scratch: a clear error, nothing enqueued
    big = torch.zeros(33 * 32 * 32, dtype=torch.float64, device="cuda")
    assert f(big.data_ptr(), big.data_ptr(), 33, 32, 32, (C.c_double * 3)(*hr), None) == -8
    assert f(big.data_ptr(), big.data_ptr(), 7, 8, 8, (C.c_double * 3)(*hr), None) == -8
    assert f(None, big.data_ptr(), 8, 8, 8, (C.c_double * 3)(*hr), None) == -1
