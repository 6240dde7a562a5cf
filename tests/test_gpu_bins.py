"""GPU parity of the image-charge solve and the energy-bin loop against the
CPU oracle, through the C ABI.

Reference behaviour covered:

* PoissonSolver::computePotential(rho, hr, zshift)       FFTPoissonSolver.cpp:287-327
  with shiftedIntGreensFunction / mirrorRhoField(Field_t&) :546-639, :667-693
* PartBunch::computeSelfFields(int bin)                   PartBunch.cpp:138-430
* calcGammas / setBinCharge                               PartBunchBase.hpp:639-683, :722-725
* the energy-bin loop of computeSpaceChargeFields          ParallelTTracker.cpp:567-578

The oracle runs in its exact mode (correctly rounded atan / log, exact
particle sums), as in test_gpu_parity.py.  Tolerances are norm-wise,
max|gpu - oracle| / max|oracle|.  The device sums the fields of all bins and
images on the mesh before one gather; the reference gathers each bin's field
and adds per particle.  The gather is linear, so the two differ by the order
of the additions only, far inside FIELD_TOL.
"""
import os

import numpy as np
import pytest

from src_b200.bunch import photoinjector_bunch

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-12
STATE_TOL = 1e-12
GOLDEN_TOL = 2e-11
MIXED_TOL = 1e-5
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(autouse=True)
def _oracle_exact(oracle):
    prev = oracle.set_threads(oracle.max_threads())
    with oracle.exact():
        yield
    oracle.set_threads(prev)


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


def test_image_potential_golden(gpu):
    g = np.load(os.path.join(GOLD, "image_n8.npz"))
    with gpu.Context((8, 8, 8)) as c:
        phi = c.compute_potential_image(g["rho"], g["hr"], float(g["zshift"]))
    assert rel(phi, g["phi"]) < GOLDEN_TOL


@pytest.mark.parametrize("nr", [(16, 16, 16), (16, 24, 32), (40, 20, 60), (64, 64, 64), (128, 128, 128)])
@pytest.mark.parametrize("zshift", [-3.3e-2, -1.0e-3, 0.0, 2.5e-3])
def test_image_potential_vs_oracle(oracle, gpu, nr, zshift):
    rng = np.random.default_rng(sum(nr))
    rho = np.abs(rng.standard_normal((nr[2], nr[1], nr[0])))
    hr = (2.7e-4, 2.9e-4, 5.1e-4)
    with gpu.Context(nr) as c:
        phi = c.compute_potential_image(rho, hr, zshift)
        # the plain solve on the same context still agrees afterwards
        phi0 = c.compute_potential(rho, hr)
    assert rel(phi, oracle.compute_potential_shifted(rho, hr, zshift)) < FIELD_TOL
    assert rel(phi0, oracle.compute_potential(rho, hr)) < FIELD_TOL


def test_image_potential_mixed(oracle, gpu):
    nr = (64, 64, 64)
    rng = np.random.default_rng(7)
    rho = np.abs(rng.standard_normal((nr[2], nr[1], nr[0])))
    hr = (2.7e-4, 2.9e-4, 5.1e-4)
    with gpu.Context(nr, precision=gpu.MIXED) as c:
        phi = c.compute_potential_image(rho, hr, -1e-2)
    assert rel(phi, oracle.compute_potential_shifted(rho, hr, -1e-2)) < MIXED_TOL


@pytest.mark.parametrize("N,nr,nbins,last", [(20_000, (16, 16, 16), 4, 4), (60_000, (32, 32, 32), 10, 10),
                                             (30_001, (16, 24, 48), 6, 3), (200_000, (64, 64, 64), 8, 8)])
def test_self_fields_binned_vs_oracle(oracle, gpu, N, nr, nbins, last):
    R, P, bins = photoinjector_bunch(N, nbins=nbins, bunch_id=N % 97)
    Q = -1e-9 / N
    prm = oracle.make_params(nr, 1e-12)
    Ef_o, Bf_o, g_o, _ = oracle.compute_self_fields_binned(prm, Q, R, P, bins, nbins, last_emitted=last)
    with gpu.Context(nr) as c:
        Ef, Bf, g = c.compute_self_fields_binned(R, P, bins, nbins, Q, 1e-12, last_emitted=last)
    # bin gammas: exact sums on both sides, one rounding, one division
    np.testing.assert_array_equal(g, g_o)
    assert rel(Ef, Ef_o) < FIELD_TOL
    assert rel(Bf, Bf_o) < FIELD_TOL


def test_self_fields_binned_linearity_full_size(gpu):
    """Size-independent property at 2e6 particles / 64^3: with equal bin
    gammas, 8 bins give the field of one bin holding every particle."""
    N = 2_000_000
    R, P, bins = photoinjector_bunch(N, nbins=8, bunch_id=11)
    P[:] = (0.0, 0.0, 1.2)
    Q = -1e-9 / N
    with gpu.Context((64, 64, 64)) as c:
        E8, B8, g8 = c.compute_self_fields_binned(R, P, bins, 8, Q, 1e-12)
        E1, B1, g1 = c.compute_self_fields_binned(R, P, np.zeros(N, np.int32), 1, Q, 1e-12)
    assert np.all(g8 == g1[0])
    assert np.linalg.norm(E8 - E1) < 1e-12 * np.linalg.norm(E1)
    assert np.linalg.norm(B8 - B1) < 1e-12 * np.linalg.norm(B1)


@pytest.mark.parametrize("N,nr,nbins,steps", [(20_000, (16, 16, 16), 4, 5), (50_000, (32, 32, 32), 6, 20)])
def test_tracking_binned_vs_oracle(oracle, gpu, N, nr, nbins, steps):
    """The step loop with energy bins (a reorder every 7 steps: the bins must
    travel with their particles)."""
    R, P, bins = photoinjector_bunch(N, nbins=nbins, bunch_id=nbins)
    Q = -1e-9 / N
    tr = oracle.OracleTracker(oracle.make_params(nr, 1e-12, ref_pz=1.0), Q)
    Ro, Po = R.copy(), P.copy()
    tr.track(Ro, Po, steps, bins=bins, nbins=nbins)
    with gpu.Context(nr) as c:
        c.upload(R, P, 1e-12, Q, oracle.electron_mass_ev(), ref_P=(0.0, 0.0, 1.0))
        c.set_energy_bins(bins, nbins)
        c.set_reorder_interval(7)
        c.track(steps)
        Rg, Pg = c.download()
        st = c.tracker_state()
        g, cnt = c.bin_gammas()
    assert rel(Rg, Ro) < STATE_TOL
    assert rel(Pg, Po) < STATE_TOL
    assert st["q_macro"] == tr.Q == Q
    assert st["path_length"] == tr.path_length
    np.testing.assert_array_equal(cnt, np.bincount(bins, minlength=nbins))
    gam = np.sqrt(1.0 + (Pg * Pg).sum(1))
    assert np.all(g > 1.0) and np.all(np.isfinite(gam))


def test_rebin_returns_to_one_solve(oracle, gpu):
    """nbins = 0 (Distribution::Rebin) gives the plain step again."""
    N, nr = 20_000, (16, 16, 16)
    R, P, bins = photoinjector_bunch(N, nbins=4, bunch_id=2)
    Q = -1e-9 / N
    tr = oracle.OracleTracker(oracle.make_params(nr, 1e-12, ref_pz=1.0), Q)
    Ro, Po = R.copy(), P.copy()
    tr.track(Ro, Po, 2, bins=bins, nbins=4)
    tr.track(Ro, Po, 3)
    with gpu.Context(nr) as c:
        c.upload(R, P, 1e-12, Q, oracle.electron_mass_ev(), ref_P=(0.0, 0.0, 1.0))
        c.set_energy_bins(bins, 4)
        c.track(2)
        c.set_energy_bins(None, 0)
        c.track(3)
        Rg, Pg = c.download()
        q = c.tracker_state()["q_macro"]
    assert rel(Rg, Ro) < STATE_TOL and rel(Pg, Po) < STATE_TOL
    assert q == tr.Q


def test_binned_errors_are_reported(gpu):
    N, nr = 5_000, (16, 16, 16)
    R, P, bins = photoinjector_bunch(N, nbins=4, bunch_id=4)
    with gpu.Context(nr) as c:
        with pytest.raises(gpu.ScgpuError) as e:
            c.set_energy_bins(bins, 4)  # no bunch yet
        assert e.value.code == -7
        c.upload(R, P, 1e-12, -1e-9 / N, 0.51099892e6, ref_P=(0.0, 0.0, 1.0))
        with pytest.raises(gpu.ScgpuError) as e:
            c.set_energy_bins(bins, 65)
        assert e.value.code == -1
        bad = bins.copy()
        bad[17] = 9
        c.set_energy_bins(bad, 4)
        with pytest.raises(gpu.ScgpuError) as e:
            c.track(1)
        assert e.value.code == -1 and "energy bin" in str(e.value)
        # the context stays usable
        c.upload(R, P, 1e-12, -1e-9 / N, 0.51099892e6, ref_P=(0.0, 0.0, 1.0))
        c.set_energy_bins(bins, 4)
        c.track(2)
