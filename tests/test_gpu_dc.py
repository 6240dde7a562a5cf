"""GPU parity of DC-beam tracking (FIELDSOLVER BCFFTZ=PERIODIC with
PartBunch::setBCForDCBeam, src/Classic/Algorithms/PartBunch.cpp:1079-1098)
against the CPU oracle, through the C ABI.

The beam is longer than its period so that particles wrap at the top of the
mesh's domain from the first step, and both z guard planes of the CIC
stencil are reached (the scatter drops their charge, the gather reads the
field's periodic images).  Tolerances as in test_gpu_parity: norm-wise
1e-12 for fields and particle state against the oracle's exact mode.
"""
import math

import numpy as np
import pytest

from src_b200.bunch import dc_bunch

pytestmark = pytest.mark.gpu

C_LIGHT = 299792458.0
FIELD_TOL = 1e-12
STATE_TOL = 1e-12
RHO_TOL = 1e-13
NR = (16, 16, 32)
LENGTH = 6e-3
FREQ = C_LIGHT / 5.7e-3          # the BEAM frequency whose period is 5.7 mm
PERIOD = C_LIGHT / FREQ           # the library's period length, c / f


@pytest.fixture(autouse=True)
def _oracle_exact(oracle):
    prev = oracle.set_threads(oracle.max_threads())
    with oracle.exact():
        yield
    oracle.set_threads(prev)


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


def dc_context(gpu, nr=NR, precision=0):
    c = gpu.Context(nr, precision=precision)
    c.set_periodic_z(True)
    c.set_beam_frequency(FREQ)
    return c


def test_dc_self_fields_vs_oracle(oracle, gpu):
    N = 40_000
    R, P = dc_bunch(N, LENGTH, bunch_id=5)
    Q = -1e-9 / N
    prm = oracle.make_params(NR, 1e-12, period=PERIOD)
    Ef_o, Bf_o, q_o, dbg = oracle.compute_self_fields(prm, Q, R, P)
    wrapped = (dbg["R"] != R).any(axis=1).sum()
    assert wrapped > 100
    with dc_context(gpu) as c:
        Ef, Bf, q = c.compute_self_fields(R, P, Q, 1e-12)
        rho, phi, E, m = c.field(gpu.FIELD_RHO), c.field(gpu.FIELD_PHI), c.field(gpu.FIELD_E), c.mesh()
    assert q == q_o
    np.testing.assert_array_equal(m["hr"], dbg["hr"])
    np.testing.assert_array_equal(m["origin"], dbg["origin"])
    assert math.isclose(m["gammaz"], dbg["gammaz"], rel_tol=1e-13)
    assert rel(rho, dbg["rho"]) < RHO_TOL
    assert rel(phi, dbg["phi"]) < FIELD_TOL
    assert rel(E, dbg["E"]) < FIELD_TOL
    assert rel(Ef, Ef_o) < FIELD_TOL
    assert rel(Bf, Bf_o) < FIELD_TOL


def _track_pair(oracle, gpu, N, nr, steps, reorder=None, precision=0):
    R, P = dc_bunch(N, LENGTH, bunch_id=6)
    Q = -1e-9 / N
    prm = oracle.make_params(nr, 1e-12, period=PERIOD)
    tr = oracle.OracleTracker(prm, Q)
    Ro, Po = R.copy(), P.copy()
    dbg = tr.track(Ro, Po, steps, want_debug=True)
    with dc_context(gpu, nr, precision) as c:
        if reorder is not None:
            c.set_reorder_interval(reorder)
        c.upload(R, P, 1e-12, Q, oracle.electron_mass_ev())
        c.track(steps)
        Rg, Pg = c.download()
        g = dict(R=Rg, P=Pg, st=c.tracker_state(), rho=c.field(gpu.FIELD_RHO), E=c.field(gpu.FIELD_E),
                 bp=c.beam_parameters())
    return dict(R=Ro, P=Po, tr=tr, dbg=dbg, R0=R), g


@pytest.mark.parametrize("N,nr,steps", [(30_000, (16, 16, 32), 10), (50_001, (32, 16, 24), 6)])
def test_dc_tracking_vs_oracle(oracle, gpu, N, nr, steps):
    o, g = _track_pair(oracle, gpu, N, nr, steps)
    assert rel(g["R"], o["R"]) < STATE_TOL
    assert rel(g["P"], o["P"]) < STATE_TOL
    assert rel(g["rho"], o["dbg"]["rho"]) < RHO_TOL
    assert rel(g["E"], o["dbg"]["E"]) < FIELD_TOL
    st, tr = g["st"], o["tr"]
    assert st["path_length"] == tr.path_length and st["t"] == tr.t and st["q_macro"] == tr.Q
    bo = oracle.beam_parameters(o["R"], o["P"])
    assert rel(g["bp"]["moments"], bo["moments"]) < 1e-12
    # the beam did wrap: its z extent stays within about one mesh domain
    span0 = np.ptp(o["R0"][:, 2])
    assert np.ptp(g["R"][:, 2]) < span0


def test_dc_tracking_independent_of_cell_order(oracle, gpu):
    """The cell reorder sorts particles of the guard plane -1 with plane 0;
    the exact sums make the result independent of the order."""
    _, a = _track_pair(oracle, gpu, 30_000, NR, 8, reorder=0)
    _, b = _track_pair(oracle, gpu, 30_000, NR, 8, reorder=2)
    np.testing.assert_array_equal(a["R"], b["R"])
    np.testing.assert_array_equal(a["P"], b["P"])


def test_dc_mixed_form_vs_plain(oracle, gpu):
    o, plain = _track_pair(oracle, gpu, 30_000, NR, 10)
    _, mixed = _track_pair(oracle, gpu, 30_000, NR, 10, precision=gpu.MIXED)
    assert rel(mixed["E"], plain["E"]) < 1e-5
    for d in range(3):
        assert math.isclose(mixed["bp"]["eps_norm"][d], plain["bp"]["eps_norm"][d], rel_tol=1e-6)
    assert rel(mixed["R"], plain["R"]) < 1e-9


def test_beam_frequency_arguments(gpu):
    with gpu.Context(NR) as c:
        for bad in (0.0, -1.0, float("nan"), float("inf")):
            with pytest.raises(gpu.ScgpuError) as e:
                c.set_beam_frequency(bad)
            assert e.value.code == -1
        c.set_beam_frequency(1.3e9)
