"""ASTRA 1D magnetostatic field maps (Astra1DMagnetoStatic.cpp, readMap
:83-160, getFieldstrength :162-196) on the host: the reader's Fourier
coefficients against an independent numpy / scipy computation of the same
recipe (natural cubic spline resampling, mirrored 2N-point sequence, DFT),
the series against the sampled field, and the off-axis expansion against
div B = 0."""
import numpy as np
import pytest

from src_b200.bunch import write_solenoid_map


@pytest.fixture(scope="module")
def sg():
    from src_b200 import scgpu
    scgpu.lib()
    return scgpu


def _recipe(z, bz, accuracy):
    from scipy.interpolate import CubicSpline
    N = len(z)
    dz = (z[-1] - z[0]) / (N - 1)
    res = np.empty(N)
    res[:-1] = CubicSpline(z, bz, bc_type="natural")(z[0] + dz * np.arange(N - 1))
    res[-1] = bz[-1]
    X = np.fft.fft(np.concatenate([res[::-1], res]))
    c = np.empty(2 * accuracy - 1)
    c[0] = X[0].real / (2 * N)
    c[1::2] = X[1:accuracy].real / N
    c[2::2] = X[1:accuracy].imag / N
    return c / np.abs(bz).max(), 2.0 * N * (z[-1] - z[0]) / (N - 1)


@pytest.mark.parametrize("jitter", [0.0, 0.3])
def test_reader_matches_recipe(sg, tmp_path, jitter):
    path = tmp_path / "sol.txt"
    z, bz = write_solenoid_map(path, accuracy=40, jitter=jitter)
    c, zb, ze, per = sg.fieldmap_astra1d(path)
    ref, per_ref = _recipe(z, bz, 40)
    assert zb == z[0] and ze == z[-1] and per == per_ref
    assert np.abs(c - ref).max() < 1e-14


def test_series_reproduces_the_map(sg, oracle, tmp_path):
    path = tmp_path / "sol.txt"
    z, bz = write_solenoid_map(path, accuracy=80, width=0.02)
    c, zb, ze, per = sg.fieldmap_astra1d(path)
    e = oracle.make_solenoid(c, zb, ze, per, 0.0, 2.0)
    pts = np.column_stack([np.zeros_like(z), np.zeros_like(z), z])[:-1]
    B = oracle.solenoid_field(e, pts)
    # 80 harmonics of the mirrored profile: the kink of the mirror at the map's
    # ends converges slowly, the interior to ~1e-4 of the peak
    err = np.abs(B[:, 2] - 2.0 * bz[:-1])
    inner = (z[:-1] > 0.05) & (z[:-1] < 0.25)
    assert err[inner].max() < 2e-4 * 2.0 and err.max() < 2e-3 * 2.0
    assert np.all(B[:, :2] == 0.0)
    # outside [zbegin, zend) an element contributes nothing
    assert np.all(oracle.solenoid_field(e, np.array([[0.0, 0.0, -1e-3], [0.0, 0.0, ze]])) == 0.0)


def test_off_axis_expansion_is_divergence_free(sg, oracle, tmp_path):
    path = tmp_path / "sol.txt"
    write_solenoid_map(path, accuracy=40)
    c, zb, ze, per = sg.fieldmap_astra1d(path)
    e = oracle.make_solenoid(c, zb, ze, per, 0.0, 1.0)
    h, r = 1e-6, 2e-3
    for zq in (0.03, 0.1, 0.27):
        f = lambda x, zz: oracle.solenoid_field(e, np.array([[x, 0.0, zz]]))[0]
        dbz = (f(r, zq + h)[2] - f(r, zq - h)[2]) / (2 * h)
        drbr = ((r + h) * f(r + h, zq)[0] - (r - h) * f(r - h, zq)[0]) / (2 * h)
        assert abs(dbz + drbr / r) < 1e-6 * max(abs(dbz), 1.0)


@pytest.mark.parametrize("text", ["AstraMagnetostatic 10 MAYBE\n0 1\n0.1 1\n0.2 1\n",
                                  "AstraElectrostatic 10\n0 1\n0.1 1\n0.2 1\n",
                                  "AstraMagnetostatic 10\n0 1\n0.1 1 3\n0.2 1\n",
                                  "AstraMagnetostatic 10\n0 1\n0.1 1\n"])
def test_reader_errors(sg, tmp_path, text):
    path = tmp_path / "bad.txt"
    path.write_text(text)
    with pytest.raises(sg.ScgpuError):
        sg.fieldmap_astra1d(path)


def test_reader_comments_and_dropped_points(sg, tmp_path):
    path = tmp_path / "sol.txt"
    path.write_text("# solenoid\nAstraMagnetostatic 3 FALSE\n\n0.0 0.5 # first\n0.1 1.0\n0.1 9.0\n0.2 0.5\n0.3 0.25\n")
    c, zb, ze, per = sg.fieldmap_astra1d(path)
    assert zb == 0.0 and ze == 0.3 and abs(per - 2 * 4 * 0.3 / 3) < 1e-15
    ref, _ = _recipe(np.array([0.0, 0.1, 0.2, 0.3]), np.array([0.5, 1.0, 0.5, 0.25]), 3)
    np.testing.assert_allclose(c, ref * 1.0, rtol=0, atol=1e-15)  # FALSE: not normalised (max |Bz| = 1 here)


# ---------------------------------------------------------------- RF cavities
# ASTRA 1D dynamic maps (Astra1DDynamic.cpp: readMap :96-185, getFieldstrength
# :192-229) and RFCavity::apply (RFCavity.cpp:232-249).

@pytest.mark.parametrize("jitter", [0.0, 0.3])
def test_dynamic_reader_matches_recipe(sg, tmp_path, jitter):
    from src_b200.bunch import write_rfcavity_map

    path = tmp_path / "cav.txt"
    z, ez = write_rfcavity_map(path, accuracy=40, jitter=jitter)
    c, zb, ze, per, f = sg.fieldmap_astra1d_dynamic(path)
    ref, per_ref = _recipe(z, ez, 40)
    assert f == 1300.0 and zb == z[0] and ze == z[-1] and per == per_ref
    assert np.abs(c - 1e6 * ref).max() < 1e-14 * 1e6   # normalised to 1 MV/m, in V/m


@pytest.mark.parametrize("text", ["AstraDynamic 10\n0 1\n0.1 1\n0.2 1\n",          # no frequency line
                                  "AstraDynamic 10\n1300 1\n0 1\n0.1 1\n0.2 1\n",  # two numbers on it
                                  "AstraMagnetostatic 10\n1300\n0 1\n0.1 1\n0.2 1\n"])
def test_dynamic_reader_errors(sg, tmp_path, text):
    path = tmp_path / "bad.txt"
    path.write_text(text)
    with pytest.raises(sg.ScgpuError):
        sg.fieldmap_astra1d_dynamic(path)


def test_rfcavity_on_axis_and_time_dependence(sg, oracle, tmp_path):
    """On axis E_z = VOLT cos(omega t + LAG) E_map(z) and B = 0; off axis
    B oscillates in quadrature (as -sin); outside the map no field."""
    from src_b200.bunch import write_rfcavity_map

    path = tmp_path / "cav.txt"
    z, ez = write_rfcavity_map(path, accuracy=80)
    c, zb, ze, per, f = sg.fieldmap_astra1d_dynamic(path)
    e = oracle.make_rfcavity(c, zb, ze, per, f, 0.0, 12.0, 1300.0, 0.3)
    w = e.omega
    for t in (0.0, 1.7e-10):
        pts = np.column_stack([np.zeros_like(z), np.zeros_like(z), z])[40:-40]
        E, B = oracle.rfcavity_field(e, pts, t)
        want = 12.0 * np.cos(w * t + 0.3) * 1e6 * ez[40:-40]
        assert np.abs(E[:, 2] - want).max() < 2e-3 * 12e6
        assert np.all(E[:, :2] == 0.0) and np.all(B == 0.0)
    p = np.array([[1e-3, -2e-3, 0.05]])
    E0, B0 = oracle.rfcavity_field(e, p, 0.0)
    E1, B1 = oracle.rfcavity_field(e, p, np.pi / 2 / w)  # a quarter period later
    assert np.any(B0 != 0.0)
    np.testing.assert_allclose(E0 / np.cos(0.3), E1 / np.cos(np.pi / 2 + 0.3), rtol=1e-9)
    np.testing.assert_allclose(B0 / np.sin(0.3), B1 / np.sin(np.pi / 2 + 0.3), rtol=1e-9)
    E, B = oracle.rfcavity_field(e, np.array([[0.0, 0.0, -1e-3], [0.0, 0.0, ze]]), 0.0)
    assert np.all(E == 0.0) and np.all(B == 0.0)


def test_rfcavity_expansion_is_divergence_free(sg, oracle, tmp_path):
    from src_b200.bunch import write_rfcavity_map

    path = tmp_path / "cav.txt"
    write_rfcavity_map(path, accuracy=40)
    c, zb, ze, per, f = sg.fieldmap_astra1d_dynamic(path)
    e = oracle.make_rfcavity(c, zb, ze, per, f, 0.0, 1.0, 1300.0, 0.0)
    h, r = 1e-6, 1e-3
    for zq in (0.03, 0.1, 0.17):
        g = lambda x, zz: oracle.rfcavity_field(e, np.array([[x, 0.0, zz]]), 0.0)[0][0]
        dez = (g(r, zq + h)[2] - g(r, zq - h)[2]) / (2 * h)
        drer = ((r + h) * g(r + h, zq)[0] - (r - h) * g(r - h, zq)[0]) / (2 * h)
        assert abs(dez + drer / r) < 1e-4 * max(abs(dez), 1e6)
