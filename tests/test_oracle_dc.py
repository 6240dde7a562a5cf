"""CPU tests of the oracle's DC-beam pieces (PartBunch::setBCForDCBeam,
src/Classic/Algorithms/PartBunch.cpp:1079-1098, chosen by TrackRun for a
field solver with periodic z, src/Track/TrackRun.cpp:899-902):

* boundp's mesh with z spanning one period (PartBunchBase.hpp:813-843);
* the periodic particle boundary along z over the mesh's domain
  [origin, origin + n h) (ParticlePeriodicBCond, ippl/src/Particle/
  ParticleBConds.h:37-45; RegionLayout::getMeshDomain, ippl/src/Region/
  RegionLayout.hpp:773-789);
* the scatter that drops the charge landing in the z guard layer and the
  gather that reads the guard layer's periodic images.

The reference has no test or fixture for this path; these check the
restatement against independent numpy statements of the same rules.
"""
import numpy as np
import pytest

from src_b200.bunch import dc_bunch

NR = (16, 16, 32)
LENGTH = 6e-3
PERIOD = 5.7e-3  # shorter than the beam: the top particles wrap


def _wrapped(oracle):
    R, _ = dc_bunch(20_000, LENGTH, bunch_id=3)
    m = oracle.boundp_dc(R, NR, 0.02, PERIOD)
    return R, m, oracle.wrap_z(R, m)


def _cic_z(z, m):
    """lower z plane and offset of each particle (IntCIC's index rules)"""
    o, h = m.origin[2], m.hr[2]
    i = np.trunc((z - o) / h).astype(np.int64)
    ngp = np.where(z >= o, i, i - 1)
    g = (ngp + 0.5) * h + o
    low = g > z
    l = np.where(low, ngp - 1, ngp)
    g = np.where(low, g - h, g)
    return l, (z - g) / h


def test_boundp_dc_mesh(oracle):
    R, _ = dc_bunch(20_000, LENGTH, bunch_id=3)
    m = oracle.boundp_dc(R, NR, 0.02, PERIOD)
    mo = oracle.boundp(R, NR, 0.02)
    for d in range(2):  # x, y exactly as for an open bunch
        assert m.hr[d] == mo.hr[d] and m.origin[d] == mo.origin[d]
        assert m.rmin[d] == mo.rmin[d] and m.rmax[d] == mo.rmax[d]
    zmin = float(R[:, 2].min())
    assert m.rmin[2] == zmin
    assert m.rmax[2] == zmin + PERIOD
    assert m.hr[2] == PERIOD / (NR[2] - 1)
    assert m.origin[2] == zmin - m.hr[2] / 2.0


def test_wrap_z_over_the_mesh_domain(oracle):
    R, m, W = _wrapped(oracle)
    lo = m.origin[2]
    hi = m.origin[2] + m.hr[2] * NR[2]
    np.testing.assert_array_equal(W[:, :2], R[:, :2])
    inside = (R[:, 2] >= lo) & (R[:, 2] < hi)
    above = R[:, 2] >= hi
    assert above.sum() > 100  # the beam is longer than the domain
    np.testing.assert_array_equal(W[inside, 2], R[inside, 2])
    np.testing.assert_array_equal(W[above, 2], lo + (R[above, 2] - hi))
    # below the domain (possible when a later step's mesh starts higher)
    T = R[:5].copy()
    T[:, 2] = lo - np.array([1e-6, 2e-5, 3e-4, 1e-3, 0.0])
    Tw = oracle.wrap_z(T, m)
    below = T[:, 2] < lo
    np.testing.assert_array_equal(Tw[below, 2], hi - (lo - T[below, 2]))
    assert Tw[~below, 2][0] == T[~below, 2][0]


def test_scatter_dc_drops_guard_layer_charge(oracle):
    _, m, W = _wrapped(oracle)
    q = -1e-15
    l, d = _cic_z(W[:, 2], m)
    assert (l == -1).any() and (l == NR[2] - 1).any()  # both guard planes are reached
    kept = np.where(l >= 0, 1 - d, 0.0) + np.where(l + 1 <= NR[2] - 1, d, 0.0)
    rho = oracle.scatter_cic(W, q, m, dc=True)
    assert abs(rho.sum() - q * kept.sum()) <= 1e-12 * abs(q) * len(W)
    assert kept.sum() < len(W)  # some charge is lost, as in the reference
    with pytest.raises(RuntimeError):  # the open scatter rejects guard-cell stencils
        oracle.scatter_cic(W, q, m)


def test_gather_dc_reads_periodic_images(oracle):
    _, m, W = _wrapped(oracle)
    rng = np.random.default_rng(4)
    E = rng.standard_normal((NR[2], NR[1], NR[0], 3))
    Ef = oracle.gather_cic(W, m, E, dc=True)
    # numpy statement: x, y as the open CIC, z planes taken modulo n
    ix = []
    dx = []
    for a in range(2):
        o, h = m.origin[a], m.hr[a]
        u = (W[:, a] - o) / h - 0.5
        la = np.floor(u).astype(np.int64)
        ix.append(la)
        dx.append(u - la)
    lz, dz = _cic_z(W[:, 2], m)
    out = np.zeros_like(Ef)
    for k in range(8):
        a0, a1, a2 = k & 1, (k >> 1) & 1, (k >> 2) & 1
        w = (dx[0] if a0 else 1 - dx[0]) * (dx[1] if a1 else 1 - dx[1]) * (dz if a2 else 1 - dz)
        zi = (lz + a2) % NR[2]
        out += w[:, None] * E[zi, ix[1] + a1, ix[0] + a0]
    assert np.max(np.abs(Ef - out)) <= 1e-13 * np.max(np.abs(E))
    top = lz == NR[2] - 1
    assert top.any()


def test_dc_self_fields_wrap_the_callers_copy_only(oracle):
    R, P = dc_bunch(20_000, LENGTH, bunch_id=3)
    R0 = R.copy()
    prm = oracle.make_params(NR, 1e-12, period=PERIOD)
    Ef, Bf, q, dbg = oracle.compute_self_fields(prm, -1e-9 / len(R), R, P)
    np.testing.assert_array_equal(R, R0)
    m = oracle.boundp_dc(R0, NR, 0.02, PERIOD)
    np.testing.assert_array_equal(dbg["R"], oracle.wrap_z(R0, m))
    assert np.all(np.isfinite(Ef)) and np.all(np.isfinite(Bf))
    # energy bins are not a DC-beam configuration
    with pytest.raises(RuntimeError):
        oracle.compute_self_fields_binned(prm, -1e-9 / len(R), R, P, np.zeros(len(R), np.int32), 1)


def test_dc_tracker_keeps_particles_in_the_period(oracle):
    """A tracked DC beam stays within one mesh domain of its lowest particle
    plus one step's drift: the wrap folds what leaves the top back in."""
    R, P = dc_bunch(20_000, LENGTH, bunch_id=3)
    prm = oracle.make_params(NR, 1e-12, period=PERIOD)
    tr = oracle.OracleTracker(prm, -1e-9 / len(R))
    for _ in range(3):
        tr.track(R, P, 2)
        span = R[:, 2].max() - R[:, 2].min()
        assert span < PERIOD * NR[2] / (NR[2] - 1) + 1e-3
