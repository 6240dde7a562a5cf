"""CPU tests of the oracle's MULTIPOLE element (src/Classic/AbsBeamline/
Multipole.cpp): the field of Multipole::computeField against the complex
statement of a straight multipole, B_y + i B_x = sum_n c_n f_n z^(n-1) for the
normal components and B_x - i B_y = -sum_n s_n f_n z^(n-1) for the skew ones
(z = x + i y; f_n = 1 for orders 1..5 and 1/(n-1)! beyond, the normalisation
of the reference's series), with the components stored as
setNormalComponent / setSkewComponent store them (:106-163); the hard edges
at 0 and L; the elliptical aperture; the reference particle's components
less their errors (:377-397).
"""
import math

import numpy as np

KN = [1.5e-3, 3.0, 200.0, 4e3, 7e4, 3e6, 2e8, 5e9]
KS = [0.0, 0.8, 50.0, 1e3, 0.0, 1e6, 0.0]


def stored(oracle, v, verr, n, skew):
    import ctypes as C
    L = oracle.lib()
    L.sco_multipole_component.restype = C.c_double
    e = C.c_double()
    c = L.sco_multipole_component(C.c_int(n), C.c_int(1 if skew else 0), C.c_double(v), C.c_double(verr), C.byref(e))
    return c, e.value


def test_component_scaling(oracle):
    # Multipole.cpp:106-163: dipole (v + e)/2 with error = itself, sextupole /2,
    # normal octupole and decapole /24, skew octupole /6, skew decapole /24
    assert stored(oracle, 2.0, 0.5, 1, False) == (1.25, 1.25)
    assert stored(oracle, 3.0, 1.0, 2, False) == (4.0, 1.0)
    assert stored(oracle, 4.0, 2.0, 3, False) == (3.0, 1.0)
    assert stored(oracle, 24.0, 24.0, 4, False) == (2.0, 1.0)
    assert stored(oracle, 12.0, 0.0, 4, True) == (2.0, 0.0)
    assert stored(oracle, 48.0, 0.0, 5, True) == (2.0, 0.0)
    assert stored(oracle, 7.0, 0.5, 6, False) == (7.5, 0.5)


def test_field_against_complex_series(oracle):
    e = oracle.make_multipole(0.0, 0.2, KN, None, KS, None)
    rng = np.random.default_rng(1)
    R = np.column_stack([rng.uniform(-0.02, 0.02, 200), rng.uniform(-0.02, 0.02, 200), rng.uniform(0, 0.2, 200)])
    B = oracle.multipole_field(e, R)
    z = R[:, 0] + 1j * R[:, 1]
    byx = np.zeros(len(R), complex)
    for n, v in enumerate(KN, start=1):
        c, _ = stored(oracle, v, 0.0, n, False)
        f = 1.0 if n <= 5 else 1.0 / math.factorial(n - 1)
        byx += c * f * z ** (n - 1)
    bxy = np.zeros(len(R), complex)
    for n, v in enumerate(KS, start=1):
        s, _ = stored(oracle, v, 0.0, n, True)
        f = 1.0 if n <= 5 else 1.0 / math.factorial(n - 1)
        bxy -= s * f * z ** (n - 1)
    scale = np.max(np.abs(B))
    assert np.max(np.abs(B[:, 1] - (byx.real - bxy.imag))) < 1e-12 * scale
    assert np.max(np.abs(B[:, 0] - (byx.imag + bxy.real))) < 1e-12 * scale
    assert np.all(B[:, 2] == 0.0)


def test_hard_edges_aperture_and_reference_particle(oracle):
    e = oracle.make_multipole(0.0, 0.1, [1e-3, 2.0], [4e-4, 0.5], [0.0, 1.0], [0.0, 0.25])
    pts = np.array([[1e-3, 2e-3, -1e-9], [1e-3, 2e-3, 0.0], [1e-3, 2e-3, 0.1], [1e-3, 2e-3, 0.1 + 1e-9],
                    [0.49, 0.0, 0.05], [0.5, 0.0, 0.05], [0.4, 0.4, 0.05]])
    B = oracle.multipole_field(e, pts)
    assert np.all(B[0] == 0) and np.all(B[3] == 0)  # outside 0 <= z <= L
    assert np.any(B[1] != 0) and np.any(B[2] != 0)  # both edges belong to the element
    assert np.any(B[4] != 0) and np.all(B[5] == 0) and np.all(B[6] == 0)  # 0.5 m elliptical aperture
    # the reference particle: components less errors; the dipole's error is
    # its whole stored value, so on axis it sees nothing
    on_axis = np.array([[0.0, 0.0, 0.05]])
    assert np.any(oracle.multipole_field(e, on_axis) != 0)
    assert np.all(oracle.multipole_field(e, on_axis, ref_particle=True) == 0)
    off = np.array([[1e-3, -2e-3, 0.05]])
    Bp, Br = oracle.multipole_field(e, off), oracle.multipole_field(e, off, ref_particle=True)
    quad, qerr = stored(oracle, 2.0, 0.5, 2, False)
    skq, skerr = stored(oracle, 1.0, 0.25, 2, True)
    dip, _ = stored(oracle, 1e-3, 4e-4, 1, False)
    assert math.isclose(Br[0, 1], (quad - qerr) * 1e-3 + (skq - skerr) * -2e-3, rel_tol=1e-14)
    assert math.isclose(Bp[0, 1], dip + quad * 1e-3 + skq * -2e-3, rel_tol=1e-14)
