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


def test_reader_keeps_leading_signs(sg, tmp_path):
    """Fieldmap::getLine cuts a line to its first and last letter, digit or
    '. - +' (Fieldmap.cpp:519-541, :802): a map starting at negative z."""
    path = tmp_path / "sol.txt"
    path.write_text("AstraMagnetostatic 3 FALSE\n-0.1 0.5\n  -0.05 1.0\n+0.0 0.5\n.05 -0.25\n")
    c, zb, ze, per = sg.fieldmap_astra1d(path)
    assert zb == -0.1 and ze == 0.05
    ref, _ = _recipe(np.array([-0.1, -0.05, 0.0, 0.05]), np.array([0.5, 1.0, 0.5, -0.25]), 3)
    np.testing.assert_allclose(c, ref * 1.0, rtol=0, atol=1e-15)


# ---------------------------------------------------------------- 2D maps
# FM2DMagnetoStatic / FM2DDynamic (src/Classic/Fields/FM2D*.cpp): the
# library's reader against the oracle's restatement, both orientations and
# normalisation flags; the oracle's bilinear field against numpy.

@pytest.mark.parametrize("orient", ["XZ", "ZX"])
@pytest.mark.parametrize("normalize", [None, True, False])
def test_2d_readers_agree(sg, oracle, tmp_path, orient, normalize):
    from src_b200.bunch import write_2d_rfcavity_map, write_2d_solenoid_map
    for kind, writer in (("s", write_2d_solenoid_map), ("c", write_2d_rfcavity_map)):
        path = tmp_path / f"{kind}.txt"
        writer(path, orient, normalize)
        a, b = sg.fieldmap_2d(path), oracle.read_map2d(path)
        for key in ("dynamic", "nz", "nr", "zbegin", "zend", "rbegin", "rend", "freq_mhz"):
            assert a[key] == b[key], key
        np.testing.assert_array_equal(a["values"], b["values"])
        assert a["dynamic"] == (kind == "c")
        if normalize is not False:  # normalised to the largest |Bz| (|Ez| in V/m) on the axis
            top = np.abs(a["values"][0, 0]).max()
            assert top == (1e6 if kind == "c" else 1.0)


def test_2d_reader_errors(sg, tmp_path):
    path = tmp_path / "bad.txt"
    for text in ("2DMagnetoStatic YZ\n0 1 1\n0 1 1\n1 0\n1 0\n1 0\n1 0\n",  # orientation
                 "2DMagnetoStatic XZ\n0 1 1\n0 1 1\n1 0\n1 0\n1 0\n",      # a value line short
                 "2DMagnetoStatic XZ\n0 1 1\n0 1 1\n1 0\n1 0\n1 0\n1 0\n1 0\n",  # one too many
                 "2DMagnetoStatic XZ MAYBE\n0 1 1\n0 1 1\n1 0\n1 0\n1 0\n1 0\n"):
        path.write_text(text)
        with pytest.raises(sg.ScgpuError):
            sg.fieldmap_2d(path)


def _bilinear(F, hz, hr, z, rr):
    iz, ir = np.floor(z / hz).astype(int), np.floor(rr / hr).astype(int)
    lz, lr = z / hz - iz, rr / hr - ir
    return ((1 - lz) * (1 - lr) * F[ir, iz] + lz * (1 - lr) * F[ir, iz + 1] + (1 - lz) * lr * F[ir + 1, iz]
            + lz * lr * F[ir + 1, iz + 1])


def test_2d_fields_against_bilinear(oracle, tmp_path):
    from src_b200.bunch import write_2d_rfcavity_map, write_2d_solenoid_map
    rng = np.random.default_rng(2)
    ps, pc = tmp_path / "s.txt", tmp_path / "c.txt"
    write_2d_solenoid_map(ps)
    write_2d_rfcavity_map(pc)
    ms, mc = oracle.read_map2d(ps), oracle.read_map2d(pc)
    es = oracle.make_solenoid2d(ms, 0.0, 0.7)
    ec = oracle.make_rfcavity2d(mc, 0.0, 20.0, 1300.0, 0.3)
    for e, m in ((es, ms), (ec, mc)):
        zmax = m["zend"] - m["zbegin"]
        R = np.column_stack([rng.uniform(-0.02, 0.02, 300), rng.uniform(-0.02, 0.02, 300),
                             m["zbegin"] + rng.uniform(0, zmax * 0.999, 300)])
        t = 1.1e-10
        E, B = oracle.element_fields(e, R, t)
        rr = np.hypot(R[:, 0], R[:, 1])
        z = R[:, 2] - m["zbegin"]
        hz, hr = zmax / (m["nz"] - 1), (m["rend"] - m["rbegin"]) / (m["nr"] - 1)
        v = m["values"]
        if m["dynamic"]:
            ez, er, bt = (_bilinear(v[c], hz, hr, z, rr) for c in range(3))
            ce, sb = 20.0 * np.cos(e.omega * t + 0.3), 20.0 * np.sin(e.omega * t + 0.3)
            np.testing.assert_allclose(E[:, 0], ce * er * R[:, 0] / rr, rtol=1e-12, atol=1e-9)
            np.testing.assert_allclose(E[:, 2], ce * ez, rtol=1e-12, atol=1e-9)
            np.testing.assert_allclose(B[:, 0], sb * bt * R[:, 1] / rr, rtol=1e-12, atol=1e-18)
            np.testing.assert_allclose(B[:, 1], -sb * bt * R[:, 0] / rr, rtol=1e-12, atol=1e-18)
        else:
            bz, br = _bilinear(v[0], hz, hr, z, rr), _bilinear(v[1], hz, hr, z, rr)
            np.testing.assert_allclose(B[:, 2], 0.7 * bz, rtol=1e-12, atol=1e-15)
            np.testing.assert_allclose(B[:, 1], 0.7 * br * R[:, 1] / rr, rtol=1e-12, atol=1e-15)
            assert np.all(E == 0)
    # outside the z range and beyond the last radial cell: no field
    out = np.array([[0.0, 0.0, ms["zend"] + 1e-6], [0.05, 0.0, 0.1]])
    assert np.all(oracle.element_fields(es, out)[1] == 0)


# ---------------------------------------------------------------- 3D maps
# FM3DDynamic (src/Classic/Fields/FM3DDynamic.cpp): the library's reader
# against the oracle's restatement, and the oracle's trilinear field against
# numpy, including the reference's edge rules.

@pytest.mark.parametrize("normalize", [None, True, False])
def test_3d_readers_agree(sg, oracle, tmp_path, normalize):
    from src_b200.bunch import write_3d_rfcavity_map
    path = tmp_path / "c3d.txt"
    write_3d_rfcavity_map(path, normalize)
    a, b = sg.fieldmap_3d(path), oracle.read_map3d(path)
    for key in ("nx", "ny", "nz", "xbegin", "xend", "ybegin", "yend", "zbegin", "zend", "freq_mhz"):
        assert a[key] == b[key], key
    np.testing.assert_array_equal(a["values"], b["values"])
    assert (a["nx"], a["ny"], a["nz"]) == (17, 13, 81)
    if normalize is not False:  # the largest |Ez| on the axis line is 1 MV/m in V/m
        assert np.abs(a["values"][2, 8, 6]).max() == 1e6


def test_3d_reader_errors(sg, tmp_path):
    path = tmp_path / "bad.txt"
    rows = "\n".join(["1 0 0 0 0 0"] * 8)
    for text in (f"3DDynamic MAYBE\n1300\n-1 1 1\n-1 1 1\n0 1 1\n{rows}\n",   # flag
                 f"3DDynamic\n1300\n-1 1 1\n-1 1 1\n0 1 1\n{rows}\n1 0 0 0 0 0\n",  # one too many
                 "3DDynamic\n1300\n-1 1 1\n-1 1 1\n0 1 1\n" + "\n".join(["1 0 0 0 0 0"] * 7) + "\n",  # short
                 f"3DDynamic\n1300\n-1 1 1\n-1 1 1\n0 1 1\n" + rows.replace("1 0 0 0 0 0", "1 0 0 0 0", 1) + "\n",
                 f"3DDynamic\n1300\n1 2 1\n-1 1 1\n0 1 1\n{rows}\n",  # axis outside the grid (normalised)
                 f"2DDynamic XZ\n0 1 1\n1300\n0 1 1\n{rows}\n"):
        path.write_text(text)
        with pytest.raises(sg.ScgpuError):
            sg.fieldmap_3d(path)


def _trilinear(F, h, X):
    u = X / h
    i = np.floor(u).astype(int)
    l = u - i
    out = 0.0
    for a in (0, 1):
        for b in (0, 1):
            for c in (0, 1):
                w = (l[:, 0] if a else 1 - l[:, 0]) * (l[:, 1] if b else 1 - l[:, 1]) * (l[:, 2] if c else 1 - l[:, 2])
                out = out + w * F[i[:, 0] + a, i[:, 1] + b, i[:, 2] + c]
    return out


def test_3d_field_against_trilinear(oracle, tmp_path):
    from src_b200.bunch import write_3d_rfcavity_map
    rng = np.random.default_rng(4)
    path = tmp_path / "c3d.txt"
    write_3d_rfcavity_map(path)
    m = oracle.read_map3d(path)
    e = oracle.make_rfcavity3d(m, 0.0, 20.0, 1300.0, 0.3)
    h = np.array([e.hx, e.hy, e.hz])
    lo = np.array([m["xbegin"], m["ybegin"], m["zbegin"]])
    # inside: below the last two grid planes of every axis
    top = lo + h * (np.array([m["nx"], m["ny"], m["nz"]]) - 2)
    R = lo + (top - lo) * rng.uniform(0, 0.999, (300, 3))
    t = 1.1e-10
    E, B = oracle.element_fields(e, R, t)
    ce, sb = 20.0 * np.cos(e.omega * t + 0.3), 20.0 * np.sin(e.omega * t + 0.3)
    v = m["values"]
    for c in range(3):
        np.testing.assert_allclose(E[:, c], ce * _trilinear(v[c], h, R - lo), rtol=1e-12, atol=1e-6)
        np.testing.assert_allclose(B[:, c], -sb * _trilinear(v[3 + c], h, R - lo), rtol=1e-12, atol=1e-18)
    assert np.abs(E).min() > 0
    # the last two planes of each axis, before the start, outside z: no field
    out = np.array([[top[0] + 1e-9, 0.0, 0.1], [0.0, top[1] + 1e-9, 0.1], [0.0, 0.0, top[2] + 1e-9],
                    [lo[0] - 1e-9, 0.0, 0.1], [0.0, 0.0, -1e-9], [0.0, 0.0, m["zend"] + 1e-6]])
    E, B = oracle.element_fields(e, out, t)
    assert np.all(E == 0) and np.all(B == 0)
