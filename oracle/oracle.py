"""ctypes front end of the CPU oracle (test infrastructure only).

The oracle restates OPAL's space-charge step in sequential FP64 C
(``oracle/sc_oracle.c``; every function there cites the reference file and
line it follows).  Only the tests, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` import this module -- as the checker, never as
the thing that is measured or shipped.

``use_reference_fft()`` switches the oracle's 1-D FFT engine to the
reference's own FFTPACK (``ippl/src/FFT/fftpack.cpp``) compiled from source
into ``oracle/_ref/libfftpack_ref.so`` by ``oracle/Makefile``.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libscoracle.so")
REF_FFT_PATH = os.path.join(HERE, "_ref", "libfftpack_ref.so")
# BorisPusher, Quaternion and CoordinateSystemTrafo of the reference, compiled
# from its sources by oracle/Makefile (refpin/refpin.cpp gives them a C ABI)
REF_PIN_PATH = os.path.join(HERE, "_ref", "librefpin.so")

_dp = C.POINTER(C.c_double)


class Mesh(C.Structure):
    _fields_ = [("nr", C.c_int * 3), ("hr", C.c_double * 3), ("origin", C.c_double * 3),
                ("rmin", C.c_double * 3), ("rmax", C.c_double * 3)]


class Trafo(C.Structure):
    _fields_ = [("origin", C.c_double * 3), ("quat", C.c_double * 4), ("M", C.c_double * 9)]


class Params(C.Structure):
    _fields_ = [("nr", C.c_int * 3), ("pad_", C.c_int), ("dh", C.c_double), ("dT", C.c_double),
                ("mass", C.c_double), ("charge", C.c_double), ("coupling", C.c_double),
                ("bz_ext", C.c_double), ("ref_pz", C.c_double), ("period", C.c_double)]


class Tracker(C.Structure):
    _fields_ = [("prm", Params), ("Q", C.c_double), ("t", C.c_double), ("path_length", C.c_double),
                ("ref_R", C.c_double * 3), ("ref_P", C.c_double * 3), ("ref_to_lab", Trafo),
                ("step", C.c_longlong)]


class Debug(C.Structure):
    _fields_ = [("rho", _dp), ("phi", _dp), ("E", _dp), ("Ef", _dp), ("Bf", _dp), ("mesh", Mesh),
                ("gammaz", C.c_double), ("hr_scaled", C.c_double * 3), ("pmean", C.c_double * 3),
                ("rot_beam_to_ref", C.c_double * 9), ("update_origin", C.c_double * 3)]


class Solenoid(C.Structure):
    """A beamline element: kind 0 SOLENOID, kind 1 RFCAVITY (1D maps), kind 2 MULTIPOLE."""
    _fields_ = [("edge", C.c_double), ("scale", C.c_double), ("zbegin", C.c_double), ("range", C.c_double),
                ("period", C.c_double), ("accuracy", C.c_int), ("kind", C.c_int), ("omega", C.c_double),
                ("phase", C.c_double), ("xlrep", C.c_double), ("nskew", C.c_int), ("map2d", C.c_int),
                ("aperture", C.c_double * 2), ("nz", C.c_int), ("nr", C.c_int), ("hz", C.c_double),
                ("hr", C.c_double), ("grid", _dp), ("map3d", C.c_int), ("nx", C.c_int), ("ny", C.c_int),
                ("pad3_", C.c_int), ("hx", C.c_double), ("hy", C.c_double), ("xbegin", C.c_double),
                ("ybegin", C.c_double), ("coefs", C.c_double * 255)]


class BeamParams(C.Structure):
    _fields_ = [(name, C.c_double * 3) for name in
                ("rmin", "rmax", "rmean", "pmean", "rrms", "prms", "eps_norm", "eps", "rprms")] + \
               [("gamma", C.c_double), ("moments", C.c_double * 27)]

    def as_dict(self):
        out = {name: np.array(getattr(self, name)) for name, _ in self._fields_ if name != "gamma"}
        out["gamma"] = float(self.gamma)
        return out


def build():
    """Compile the oracle (and oracle/_ref when the reference tree is present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None
_ref_fft = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.sco_const_c.restype = C.c_double
        L.sco_const_electron_mass_ev.restype = C.c_double
        L.sco_const_coupling.restype = C.c_double
        L.sco_sum_gamma.restype = C.c_double
        assert L.sco_sizeof_tracker() == C.sizeof(Tracker)
        assert L.sco_sizeof_debug() == C.sizeof(Debug)
        assert L.sco_sizeof_beam_params() == C.sizeof(BeamParams)
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def reference_fft_available():
    return os.path.exists(REF_FFT_PATH)


def use_reference_fft(on=True):
    """Route the oracle's 1-D transforms through the reference's FFTPACK."""
    global _ref_fft
    L = lib()
    if not on:
        L.sco_set_fft_engine(None, None, None, None, None, None)
        return
    if _ref_fft is None:
        _ref_fft = C.CDLL(REF_FFT_PATH)
    fn = [C.cast(getattr(_ref_fft, name), C.c_void_p) for name in
          ("cffti", "cfftf", "cfftb", "rffti", "rfftf", "rfftb")]
    L.sco_set_fft_engine(*fn)


def fft_engine_is_own():
    return bool(lib().sco_fft_engine_is_own())


def set_threads(n):
    """OpenMP threads of the oracle's particle and grid loops; returns the
    previous count."""
    L = lib()
    prev = int(L.sco_get_threads())
    L.sco_set_threads(C.c_int(int(n)))
    return prev


def max_threads():
    return int(lib().sco_max_threads())


def set_exact(on=True):
    """Exact mode: correctly rounded atan / log in the Green's function
    (quad precision) and order-independent exact particle sums (terms
    truncated at 2^-72, 128-bit integer addition, one rounding) instead of
    the reference's libm calls and storage-order sums.  Returns the previous
    setting."""
    L = lib()
    prev = bool(L.sco_get_exact())
    L.sco_set_exact(C.c_int(1 if on else 0))
    return prev


class exact:
    """Context manager: the oracle in exact mode inside."""

    def __init__(self, on=True):
        self.on = on

    def __enter__(self):
        self.prev = set_exact(self.on)
        return self

    def __exit__(self, *exc):
        set_exact(self.prev)
        return False


# ---------------------------------------------------------------- constants
def c_light():
    return lib().sco_const_c()


def electron_mass_ev():
    return lib().sco_const_electron_mass_ev()


def coupling():
    return lib().sco_const_coupling()


# ---------------------------------------------------------------- functions
def fft1d(kind, data):
    """kind: 0 cfftf, 1 cfftb, 2 rfftf, 3 rfftb (FFTPACK semantics)."""
    d = _f64(data).copy()
    n = d.size // 2 if kind < 2 else d.size
    lib().sco_fft1d(C.c_int(kind), C.c_longlong(n), _ptr(d))
    return d


def fft3d_r2c(real):
    """real: array [L2, L1, L0] (x fastest) -> complex [L2, L1, L0//2+1]."""
    r = _f64(real)
    L = (C.c_int * 3)(r.shape[2], r.shape[1], r.shape[0])
    out = np.empty((r.shape[0], r.shape[1], r.shape[2] // 2 + 1), dtype=np.complex128)
    lib().sco_fft3d_r2c(L, _ptr(r), out.ctypes.data_as(_dp))
    return out


def fft3d_c2r(spec, L0):
    s = np.ascontiguousarray(spec, dtype=np.complex128).copy()
    L = (C.c_int * 3)(L0, s.shape[1], s.shape[0])
    out = np.empty((s.shape[0], s.shape[1], L0), dtype=np.float64)
    lib().sco_fft3d_c2r(L, s.ctypes.data_as(_dp), _ptr(out))
    return out


def igf(nr, hr):
    """Doubled, mirrored integrated Green's function, array [2nz, 2ny, 2nx]."""
    G = np.empty((2 * nr[2], 2 * nr[1], 2 * nr[0]), dtype=np.float64)
    lib().sco_igf((C.c_int * 3)(*nr), (C.c_double * 3)(*hr), _ptr(G))
    return G


def compute_potential(rho, hr):
    """FFTPoissonSolver::computePotential: rho [nz, ny, nx] -> convolution."""
    r = _f64(rho).copy()
    nr = (C.c_int * 3)(r.shape[2], r.shape[1], r.shape[0])
    rc = lib().sco_compute_potential(nr, _ptr(r), (C.c_double * 3)(*hr))
    if rc:
        raise RuntimeError(f"sco_compute_potential failed: {rc}")
    return r


def make_solenoid(coefs, zbegin, zend, period, edge, ks):
    e = Solenoid()
    c = np.asarray(coefs, dtype=np.float64)
    e.edge, e.scale, e.zbegin, e.range, e.period = edge, ks, zbegin, zend - zbegin, period
    e.accuracy = (c.size + 1) // 2
    e.coefs[:c.size] = list(c)
    return e


def make_rfcavity(coefs, zbegin, zend, period, freq_map_mhz, edge, volt, freq_mhz, lag):
    """RFCAVITY (OpalCavity.cpp:150-195, RFCavity::initialise :286-310): the
    element's omega = 1e6 * two_pi * FREQ unless it differs from the map's by
    more than 1 %; the off-axis wave number from the map's frequency."""
    e = make_solenoid(coefs, zbegin, zend, period, edge, volt)
    two_pi = 2 * 3.14159265358979323846
    omega_map = freq_map_mhz * (two_pi * 1e6)
    omega = 1e6 * two_pi * freq_mhz
    if abs((omega - omega_map) / omega) > 0.01:
        omega = omega_map
    e.kind, e.omega, e.phase, e.xlrep = 1, omega, lag, omega_map / c_light()
    return e


def make_multipole(elemedge, length, kn=(), dkn=None, ks=(), dks=None, aperture=(0.5, 0.5)):
    """MULTIPOLE (OpalMultipole::update, OpalMultipole.cpp:127-166): the
    components stored as Multipole::setNormalComponent / setSkewComponent do."""
    e = Solenoid()
    e.kind, e.edge, e.range = 2, elemedge, length
    nn, ns = len(kn), len(ks)
    e.accuracy, e.nskew = nn, ns
    e.aperture[0], e.aperture[1] = aperture
    L = lib()
    L.sco_multipole_component.restype = C.c_double
    err = C.c_double()
    for i in range(nn):
        v = L.sco_multipole_component(C.c_int(i + 1), C.c_int(0), C.c_double(kn[i]),
                                      C.c_double(0.0 if dkn is None else dkn[i]), C.byref(err))
        e.coefs[i], e.coefs[nn + i] = v, err.value
    for i in range(ns):
        v = L.sco_multipole_component(C.c_int(i + 1), C.c_int(1), C.c_double(ks[i]),
                                      C.c_double(0.0 if dks is None else dks[i]), C.byref(err))
        e.coefs[2 * nn + i], e.coefs[2 * nn + ns + i] = v, err.value
    return e


def read_map2d(path):
    """A 2D (r, z) map as FM2DMagnetoStatic / FM2DDynamic read it
    (FM2DMagnetoStatic.cpp:14-155, FM2DDynamic.cpp:15-170), restated: dict
    with dynamic, nz, nr (grid points), zbegin, zend, rbegin, rend [m],
    freq_mhz and values [component, r, z] (Bz, Br or Ez, Er [V/m], Bt [T])."""
    keep = set(".-+\x89")

    def content(f):  # Fieldmap::getLine: cut to the first and last letter, digit, . - +
        for raw in f:
            line = raw.split("#", 1)[0]
            idx = [i for i, ch in enumerate(line) if ch.isalnum() or ch in keep]
            if idx:
                yield line[idx[0]:idx[-1] + 1]
    with open(path) as f:
        lines = list(content(f))
    head = lines[0].split()
    dynamic = head[0].startswith("2DDy")
    if not dynamic and not head[0].startswith("2DMa"):
        raise ValueError("not a 2D map")
    normalize = True
    if len(head) > 2:
        normalize = head[2].upper() == "TRUE"
    swap = head[1] == "ZX"
    pos = 1

    def rng():
        nonlocal pos
        a, b, n = lines[pos].split()
        pos += 1
        return float(a), float(b), int(n)
    freq = 0.0
    if swap:
        rb, re_, nri = rng()
        if dynamic:
            freq = float(lines[pos]); pos += 1
        zb, ze, nzi = rng()
    else:
        zb, ze, nzi = rng()
        if dynamic:
            freq = float(lines[pos]); pos += 1
        rb, re_, nri = rng()
    nz, nr = nzi + 1, nri + 1
    nc = 3 if dynamic else 2
    v = np.zeros((nc, nr, nz))
    rows = [[float(x) for x in l.split()] for l in lines[pos:pos + nz * nr]]
    k = 0
    if swap:
        for i in range(nz):
            for j in range(nr):
                r = rows[k]; k += 1
                v[1, j, i], v[0, j, i] = r[0], r[1]
                if dynamic:
                    v[2, j, i] = r[2]
    else:
        for j in range(nr):
            for i in range(nz):
                r = rows[k]; k += 1
                v[0, j, i], v[1, j, i] = r[0], r[1]
                if dynamic:
                    v[2, j, i] = r[3]
    amax = float(np.max(np.abs(v[0, 0, :]))) if normalize else 1.0
    if dynamic:
        mu_0 = 1.256637061e-06
        v[0] *= 1.e6 / amax
        v[1] *= 1.e6 / amax
        v[2] *= mu_0 / amax
    elif normalize:
        v[0] /= amax
        v[1] /= amax
    return dict(dynamic=dynamic, nz=nz, nr=nr, zbegin=zb / 100.0, zend=ze / 100.0, rbegin=rb / 100.0,
                rend=re_ / 100.0, freq_mhz=freq, values=v)


def _attach_map2d(e, m):
    grid = np.ascontiguousarray(m["values"], dtype=np.float64)
    e.map2d, e.nz, e.nr = 1, m["nz"], m["nr"]
    e.hz = (m["zend"] - m["zbegin"]) / (m["nz"] - 1)
    e.hr = (m["rend"] - m["rbegin"]) / (m["nr"] - 1)
    e.grid = _ptr(grid)
    e.zbegin, e.range = m["zbegin"], m["zend"] - m["zbegin"]
    e._keep = grid  # the grid must outlive the element
    return e


def make_solenoid2d(m, edge, ks):
    """SOLENOID with a 2D magnetostatic map (read_map2d) at ELEMEDGE, KS [T]."""
    e = Solenoid()
    e.kind, e.edge, e.scale = 0, edge, ks
    return _attach_map2d(e, m)


def make_rfcavity2d(m, edge, volt, freq_mhz, lag):
    """RFCAVITY with a 2D dynamic map (read_map2d): VOLT [MV/m], FREQ [MHz],
    LAG [rad]; the map's frequency replaces FREQ beyond 1 % (RFCavity.cpp:294-305)."""
    e = Solenoid()
    two_pi = 2 * 3.14159265358979323846
    omega_map = m["freq_mhz"] * (two_pi * 1e6)
    omega = 1e6 * two_pi * freq_mhz
    if abs((omega - omega_map) / omega) > 0.01:
        omega = omega_map
    e.kind, e.edge, e.scale, e.omega, e.phase = 1, edge, volt, omega, lag
    return _attach_map2d(e, m)


def read_map3d(path):
    """A 3D dynamic map as FM3DDynamic reads it (FM3DDynamic.cpp:17-220),
    restated: dict with nx, ny, nz (grid points), xbegin, xend, ybegin, yend,
    zbegin, zend [m], freq_mhz and values [component, x, y, z] (Ex, Ey, Ez
    [V/m], Bx, By, Bz [T]), normalised to the largest |Ez| on the grid line
    nearest the axis unless the header says FALSE."""
    keep = set(".-+\x89")
    with open(path) as f:
        lines = []
        for raw in f:  # Fieldmap::getLine
            line = raw.split("#", 1)[0]
            idx = [i for i, ch in enumerate(line) if ch.isalnum() or ch in keep]
            if idx:
                lines.append(line[idx[0]:idx[-1] + 1])
    head = lines[0].split()
    if not head[0].startswith("3DDy"):
        raise ValueError("not a 3D dynamic map")
    normalize = len(head) < 2 or head[1].upper() == "TRUE"
    freq = float(lines[1])
    (xb, xe, nxi), (yb, ye, nyi), (zb, ze, nzi) = [(float(a), float(b), int(n)) for a, b, n in
                                                   (l.split() for l in lines[2:5])]
    nx, ny, nz = nxi + 1, nyi + 1, nzi + 1
    rows = np.array([[float(x) for x in l.split()] for l in lines[5:5 + nx * ny * nz]])
    v = np.ascontiguousarray(rows.T.reshape(6, nx, ny, nz))
    xb, xe, yb, ye, zb, ze = (q / 100.0 for q in (xb, xe, yb, ye, zb, ze))
    hx, hy = (xe - xb) / nxi, (ye - yb) / nyi
    ezmax = 1.0
    if normalize:
        ix = int(math.ceil(-xb / hx))
        if ix * hx + xb > 0.5:
            ix -= 1
        iy = int(math.ceil(-yb / hy))
        if iy * hy + yb > 0.5:
            iy -= 1
        ezmax = float(np.max(np.abs(v[2, ix, iy, :])))
    mu_0 = 1.256637061e-06
    v[:3] *= 1e6 / ezmax
    v[3:] *= mu_0 / ezmax
    return dict(nx=nx, ny=ny, nz=nz, xbegin=xb, xend=xe, ybegin=yb, yend=ye, zbegin=zb, zend=ze, freq_mhz=freq,
                values=v)


def make_rfcavity3d(m, edge, volt, freq_mhz, lag):
    """RFCAVITY with a 3D dynamic map (read_map3d): VOLT [MV/m], FREQ [MHz],
    LAG [rad]; the map's frequency replaces FREQ beyond 1 % (RFCavity.cpp:294-305)."""
    e = Solenoid()
    two_pi = 2 * 3.14159265358979323846
    omega_map = m["freq_mhz"] * (two_pi * 1e6)
    omega = 1e6 * two_pi * freq_mhz
    if abs((omega - omega_map) / omega) > 0.01:
        omega = omega_map
    e.kind, e.edge, e.scale, e.omega, e.phase = 1, edge, volt, omega, lag
    grid = np.ascontiguousarray(m["values"], dtype=np.float64)
    e.map3d, e.nx, e.ny, e.nz = 1, m["nx"], m["ny"], m["nz"]
    e.hx = (m["xend"] - m["xbegin"]) / (m["nx"] - 1)
    e.hy = (m["yend"] - m["ybegin"]) / (m["ny"] - 1)
    e.hz = (m["zend"] - m["zbegin"]) / (m["nz"] - 1)
    e.xbegin, e.ybegin = m["xbegin"], m["ybegin"]
    e.grid = _ptr(grid)
    e.zbegin, e.range = m["zbegin"], m["zend"] - m["zbegin"]
    e._keep = grid  # the grid must outlive the element
    return e


def element_fields(element, R, t=0.0):
    """E, B of one SOLENOID / RFCAVITY element with a 2D or 3D map at points R (element frame)."""
    R = _f64(R)
    E, B = np.zeros_like(R), np.zeros_like(R)
    for i in range(R.shape[0]):
        e, b = (C.c_double * 3)(), (C.c_double * 3)()
        if element.kind == 1 and element.map3d:
            lib().sco_rfcavity3d_field(C.byref(element), R[i].ctypes.data_as(_dp), C.c_double(t), e, b)
        elif element.kind == 1:
            lib().sco_rfcavity2d_field(C.byref(element), R[i].ctypes.data_as(_dp), C.c_double(t), e, b)
        else:
            lib().sco_solenoid2d_field(C.byref(element), R[i].ctypes.data_as(_dp), b)
        E[i], B[i] = list(e), list(b)
    return E, B


def multipole_field(element, R, ref_particle=False):
    """B [T] of one MULTIPOLE at points R (n x 3, element frame)."""
    R = _f64(R)
    out = np.zeros_like(R)
    for i in range(R.shape[0]):
        b = (C.c_double * 3)()
        lib().sco_multipole_field(C.byref(element), R[i].ctypes.data_as(_dp), C.c_int(1 if ref_particle else 0), b)
        out[i] = list(b)
    return out


def rfcavity_field(element, R, t):
    """E [V/m] and B [T] of one RF cavity at points R (element frame), time t."""
    R = _f64(R)
    E, B = np.zeros_like(R), np.zeros_like(R)
    for i in range(R.shape[0]):
        e, b = (C.c_double * 3)(), (C.c_double * 3)()
        lib().sco_rfcavity_field(C.byref(element), R[i].ctypes.data_as(_dp), C.c_double(t), e, b)
        E[i], B[i] = list(e), list(b)
    return E, B


_elements_keep = []


def set_solenoids(elements):
    """SOLENOID / RFCAVITY / MULTIPOLE elements applied by the tracker
    (computeExternalFields)."""
    global _elements_keep
    _elements_keep = list(elements)  # their 2D grids stay alive while the tracker uses them
    arr = (Solenoid * max(len(elements), 1))(*elements)
    rc = lib().sco_set_solenoids(arr, C.c_int(len(elements)))
    if rc:
        raise RuntimeError(f"sco_set_solenoids failed: {rc}")


def solenoid_field(element, R):
    """B [T] of one element at points R (n x 3, element frame)."""
    R = _f64(R)
    out = np.empty_like(R)
    for i in range(R.shape[0]):
        b = (C.c_double * 3)()
        lib().sco_solenoid_field(C.byref(element), R[i].ctypes.data_as(_dp), b)
        out[i] = list(b)
    return out


def igf_periodic_z(nr, hr):
    """Green's function of the periodic-z solver, grid [nz, 2ny, 2nx]."""
    G = np.empty((nr[2], 2 * nr[1], 2 * nr[0]), dtype=np.float64)
    lib().sco_igf_periodic_z((C.c_int * 3)(*nr), (C.c_double * 3)(*hr), _ptr(G))
    return G


def compute_potential_periodic_z(rho, hr):
    """computePotential with BCFFTZ=PERIODIC: open in x, y, cyclic along z."""
    r = _f64(rho).copy()
    nr = (C.c_int * 3)(r.shape[2], r.shape[1], r.shape[0])
    rc = lib().sco_compute_potential_periodic_z(nr, _ptr(r), (C.c_double * 3)(*hr))
    if rc:
        raise RuntimeError(f"sco_compute_potential_periodic_z failed: {rc}")
    return r


def igf_shifted(nr, hr, zshift):
    """Shifted integrated Green's function of the image charge, doubled grid
    [2nz, 2ny, 2nx] (mirrored in x and y only)."""
    G = np.empty((2 * nr[2], 2 * nr[1], 2 * nr[0]), dtype=np.float64)
    lib().sco_igf_shifted((C.c_int * 3)(*nr), (C.c_double * 3)(*hr), C.c_double(zshift), _ptr(G))
    return G


def compute_potential_shifted(rho, hr, zshift):
    """FFTPoissonSolver::computePotential(rho, hr, zshift): the image-charge
    convolution of rho [nz, ny, nx], read back with z flipped."""
    r = _f64(rho).copy()
    nr = (C.c_int * 3)(r.shape[2], r.shape[1], r.shape[0])
    rc = lib().sco_compute_potential_shifted(nr, _ptr(r), (C.c_double * 3)(*hr), C.c_double(zshift))
    if rc:
        raise RuntimeError(f"sco_compute_potential_shifted failed: {rc}")
    return r


def bin_gammas(P, bins, nbins):
    """calcGammas: mean gamma per energy bin (1 for an empty bin) and counts."""
    P = _f64(P)
    b = np.ascontiguousarray(bins, dtype=np.int32)
    g = np.empty(nbins, dtype=np.float64)
    cnt = np.empty(nbins, dtype=np.int64)
    rc = lib().sco_bin_gammas(C.c_longlong(P.shape[0]), _ptr(P), b.ctypes.data_as(C.POINTER(C.c_int)),
                              C.c_int(nbins), _ptr(g), cnt.ctypes.data_as(C.POINTER(C.c_longlong)))
    if rc:
        raise RuntimeError(f"sco_bin_gammas failed: {rc}")
    return g, cnt


def compute_self_fields_binned(params, qi, R, P, bins, nbins, last_emitted=None):
    """The energy-bin loop of computeSpaceChargeFields on a beam-frame bunch:
    returns (Ef, Bf, bin gammas, debug dict with the mesh)."""
    R = _f64(R)
    P = _f64(P)
    n = R.shape[0]
    b = np.ascontiguousarray(bins, dtype=np.int32)
    Ef = np.empty_like(R)
    Bf = np.empty_like(R)
    g = np.empty(nbins, dtype=np.float64)
    dbg = Debug()
    le = nbins if last_emitted is None else last_emitted
    rc = lib().sco_compute_self_fields_binned(C.byref(params), C.c_double(qi), C.c_longlong(n), _ptr(R), _ptr(P),
                                              b.ctypes.data_as(C.POINTER(C.c_int)), C.c_int(nbins), C.c_int(le),
                                              _ptr(Ef), _ptr(Bf), _ptr(g), C.byref(dbg))
    if rc:
        raise RuntimeError(f"compute_self_fields_binned failed: {rc}")
    return Ef, Bf, g, _debug_dict(dbg, {}, list(params.nr))


def neg_grad_scaled(phi, h, gammaz):
    p = _f64(phi)
    nr = (C.c_int * 3)(p.shape[2], p.shape[1], p.shape[0])
    E = np.empty(p.shape + (3,), dtype=np.float64)
    lib().sco_neg_grad_scaled(nr, _ptr(p), (C.c_double * 3)(*h), C.c_double(gammaz), _ptr(E))
    return E


def boundp(R, nr, dh):
    R = _f64(R)
    m = Mesh()
    rc = lib().sco_boundp(C.c_longlong(R.shape[0]), _ptr(R), (C.c_int * 3)(*nr), C.c_double(dh), C.byref(m))
    if rc:
        raise RuntimeError(f"boundp failed: {rc}")
    return m


def boundp_dc(R, nr, dh, period):
    """boundp of a DC beam: z spans one period from the lowest particle."""
    R = _f64(R)
    m = Mesh()
    rc = lib().sco_boundp_dc(C.c_longlong(R.shape[0]), _ptr(R), (C.c_int * 3)(*nr), C.c_double(dh),
                             C.c_double(period), C.byref(m))
    if rc:
        raise RuntimeError(f"boundp_dc failed: {rc}")
    return m


def wrap_z(R, mesh):
    """The periodic particle boundary along z over the mesh's domain."""
    R = _f64(R).copy()
    lib().sco_wrap_z(C.c_longlong(R.shape[0]), _ptr(R), C.byref(mesh))
    return R


def scatter_cic(R, q, mesh, dc=False):
    R = _f64(R)
    nr = list(mesh.nr)
    rho = np.zeros((nr[2], nr[1], nr[0]), dtype=np.float64)
    fn = lib().sco_scatter_cic_dc if dc else lib().sco_scatter_cic
    rc = fn(C.c_longlong(R.shape[0]), _ptr(R), C.c_double(q), C.byref(mesh), _ptr(rho))
    if rc:
        raise RuntimeError(f"scatter failed: {rc}")
    return rho


def gather_cic(R, mesh, E, dc=False):
    R = _f64(R)
    E = _f64(E)
    Ef = np.empty_like(R)
    fn = lib().sco_gather_cic_dc if dc else lib().sco_gather_cic
    rc = fn(C.c_longlong(R.shape[0]), _ptr(R), C.byref(mesh), _ptr(E), _ptr(Ef))
    if rc:
        raise RuntimeError(f"gather failed: {rc}")
    return Ef


def push(R, P, dt):
    R = _f64(R).copy()
    P = _f64(P)
    lib().sco_push(C.c_longlong(R.shape[0]), _ptr(R), _ptr(P), C.c_double(dt))
    return R


def kick(P, Ef, Bf, dt, mass, charge):
    P = _f64(P).copy()
    lib().sco_kick(C.c_longlong(P.shape[0]), _ptr(P), _ptr(_f64(Ef)), _ptr(_f64(Bf)), C.c_double(dt),
                   C.c_double(mass), C.c_double(charge))
    return P


def beam_parameters(R, P):
    bp = BeamParams()
    R = _f64(R)
    P = _f64(P)
    lib().sco_beam_parameters(C.c_longlong(R.shape[0]), _ptr(R), _ptr(P), C.byref(bp))
    return bp.as_dict()


def make_params(nr, dT, dh=0.02, bz_ext=0.0, ref_pz=10.0, mass=None, charge=-1.0, period=0.0):
    """Solver and tracker parameters; period > 0 makes the bunch a DC beam
    (periodic z) with that period length [m]."""
    p = Params()
    p.nr = (C.c_int * 3)(*nr)
    p.dh = dh
    p.dT = dT
    p.mass = electron_mass_ev() if mass is None else mass
    p.charge = charge
    p.coupling = coupling()
    p.bz_ext = bz_ext
    p.ref_pz = ref_pz
    p.period = period
    return p


def compute_self_fields(params, Q, R, P, want_grids=True):
    """PartBunch::computeSelfFields on a bunch in the beam frame.
    Returns (Ef, Bf, Q_after, debug dict); for a DC beam the debug dict's
    "R" holds the positions after the periodic boundary (the caller's R is
    not changed)."""
    R = _f64(R).copy()
    P = _f64(P)
    n = R.shape[0]
    nr = list(params.nr)
    M = nr[0] * nr[1] * nr[2]
    Ef = np.empty_like(R)
    Bf = np.empty_like(R)
    dbg = Debug()
    grids = {}
    if want_grids:
        grids = {"rho": np.empty(M), "phi": np.empty(M), "E": np.empty(3 * M)}
        dbg.rho, dbg.phi, dbg.E = _ptr(grids["rho"]), _ptr(grids["phi"]), _ptr(grids["E"])
    q = C.c_double(Q)
    rc = lib().sco_compute_self_fields(C.byref(params), C.byref(q), C.c_longlong(n), _ptr(R), _ptr(P),
                                       _ptr(Ef), _ptr(Bf), C.byref(dbg))
    if rc:
        raise RuntimeError(f"compute_self_fields failed: {rc}")
    out = _debug_dict(dbg, grids, nr)
    out["R"] = R
    return Ef, Bf, q.value, out


def _debug_dict(dbg, grids, nr):
    out = {
        "hr": np.array(dbg.mesh.hr), "origin": np.array(dbg.mesh.origin),
        "rmin": np.array(dbg.mesh.rmin), "rmax": np.array(dbg.mesh.rmax),
        "gammaz": float(dbg.gammaz), "hr_scaled": np.array(dbg.hr_scaled),
        "pmean": np.array(dbg.pmean), "rot_beam_to_ref": np.array(dbg.rot_beam_to_ref).reshape(3, 3),
    }
    shape = (nr[2], nr[1], nr[0])
    for k, v in grids.items():
        out[k] = v.reshape(shape + ((3,) if k == "E" else ()))
    return out


class OracleTracker:
    """ParallelTTracker step loop restated on the CPU (sequential FP64)."""

    def __init__(self, params, Q):
        self.tr = Tracker()
        lib().sco_tracker_init(C.byref(self.tr), C.byref(params), C.c_double(Q))

    @property
    def Q(self):
        return self.tr.Q

    @property
    def t(self):
        return self.tr.t

    @property
    def path_length(self):
        return self.tr.path_length

    @property
    def ref_R(self):
        return np.array(self.tr.ref_R)

    @property
    def ref_P(self):
        return np.array(self.tr.ref_P)

    def track(self, R, P, nsteps, want_debug=False, bins=None, nbins=0, last_emitted=None):
        """Advance R, P (N x 3, updated in place) by nsteps.  With want_debug
        the last step's grids and fields are returned.  With bins (one
        energy bin per particle, nbins bins) the self fields are the
        energy-bin loop with image charges."""
        assert R.dtype == np.float64 and R.flags.c_contiguous
        assert P.dtype == np.float64 and P.flags.c_contiguous
        n = R.shape[0]
        dbgp = None
        grids = {}
        nr = list(self.tr.prm.nr)
        if want_debug:
            M = nr[0] * nr[1] * nr[2]
            grids = {"rho": np.empty(M), "phi": np.empty(M), "E": np.empty(3 * M),
                     "Ef": np.empty(3 * n), "Bf": np.empty(3 * n)}
            dbg = Debug()
            dbg.rho, dbg.phi, dbg.E = _ptr(grids["rho"]), _ptr(grids["phi"]), _ptr(grids["E"])
            dbg.Ef, dbg.Bf = _ptr(grids["Ef"]), _ptr(grids["Bf"])
            dbgp = C.byref(dbg)
        if bins is None:
            rc = lib().sco_track(C.byref(self.tr), C.c_longlong(n), _ptr(R), _ptr(P), C.c_int(nsteps), dbgp)
        else:
            b = np.ascontiguousarray(bins, dtype=np.int32)
            le = nbins if last_emitted is None else last_emitted
            rc = lib().sco_track_binned(C.byref(self.tr), C.c_longlong(n), _ptr(R), _ptr(P),
                                        b.ctypes.data_as(C.POINTER(C.c_int)), C.c_int(nbins), C.c_int(le),
                                        C.c_int(nsteps), dbgp)
        if rc:
            raise RuntimeError(f"sco_track failed: {rc}")
        if not want_debug:
            return None
        ef = grids.pop("Ef").reshape(n, 3)
        bf = grids.pop("Bf").reshape(n, 3)
        out = _debug_dict(dbg, grids, nr)
        out["Ef"], out["Bf"] = ef, bf
        out["update_origin"] = np.array(dbg.update_origin)
        return out


# ---------------------------------------------------------------- pinning
# The oracle's frame and pusher functions beside the reference's own
# (oracle/_ref/librefpin.so), on the same inputs, one case per row.

_ref_pin = None


def reference_pin_available():
    return os.path.exists(REF_PIN_PATH)


def reference_pin():
    """The reference's BorisPusher / Quaternion / CoordinateSystemTrafo
    behind a C ABI (None when oracle/_ref was not built)."""
    global _ref_pin
    if _ref_pin is None and reference_pin_available():
        _ref_pin = C.CDLL(REF_PIN_PATH)
    return _ref_pin


def _rows(fn, *arrays, out_shapes):
    """Calls fn(row pointers..., out pointers...) for every row."""
    n = len(arrays[0])
    ins = [_f64(a) for a in arrays]
    outs = [np.zeros((n,) + sh) for sh in out_shapes]
    for i in range(n):
        fn(*[_ptr(a[i]) for a in ins], *[_ptr(o[i]) for o in outs])
    return outs


def pin_cases_oracle(cases):
    """The oracle's answers for the pinning cases (see tests/golden/make_golden.py)."""
    L = lib()
    c = cases
    out = {}
    P = _f64(c["kick_P"]).copy()
    L.sco_kick(C.c_longlong(len(P)), _ptr(P), _ptr(_f64(c["kick_Ef"])), _ptr(_f64(c["kick_Bf"])),
               C.c_double(float(c["dt"])), C.c_double(float(c["mass"])), C.c_double(float(c["charge"])))
    out["kick"] = P
    R = _f64(c["push_R"]).copy()
    L.sco_push(C.c_longlong(len(R)), _ptr(R), _ptr(_f64(c["push_P"])), C.c_double(float(c["dt"])))
    out["push"] = R

    def quat(u, ref, q):
        L.sco_get_quaternion(u, ref, q)
    out["quaternion"], = _rows(quat, c["quat_u"], c["quat_ref"], out_shapes=[(4,)])

    def rotmat(q, M):
        t = Trafo()
        L.sco_trafo_make(C.byref(t), _ptr(np.zeros(3)), q)
        C.memmove(M, t.M, 9 * 8)
    out["rotation_matrix"], = _rows(rotmat, c["rotmat_quat"], out_shapes=[(9,)])
    out["quaternion_rotate"], = _rows(L.sco_quat_rotate, c["trafo_quat"], c["trafo_r"], out_shapes=[(3,)])

    def make(o, q):
        t = Trafo()
        L.sco_trafo_make(C.byref(t), o, q)
        return t

    def transform(o, q, r, res):
        t = make(o, q)
        L.sco_trafo_transform_to(C.byref(t), r, res)

    def rotate(o, q, r, res):
        t = make(o, q)
        L.sco_trafo_rotate_to(C.byref(t), r, res)

    def inverted(o, q, oo, qo):
        t = make(o, q)
        L.sco_trafo_invert(C.byref(t))
        C.memmove(oo, t.origin, 24)
        C.memmove(qo, t.quat, 32)

    def compose(lo, lq, ro, rq, oo, qo):
        t, r = make(lo, lq), make(ro, rq)
        L.sco_trafo_compose(C.byref(t), C.byref(r))
        C.memmove(oo, t.origin, 24)
        C.memmove(qo, t.quat, 32)
    out["transform_to"], = _rows(transform, c["trafo_origin"], c["trafo_quat"], c["trafo_r"], out_shapes=[(3,)])
    out["rotate_to"], = _rows(rotate, c["trafo_origin"], c["trafo_quat"], c["trafo_r"], out_shapes=[(3,)])
    out["inverted_origin"], out["inverted_quat"] = _rows(inverted, c["trafo_origin"], c["trafo_quat"],
                                                         out_shapes=[(3,), (4,)])
    out["compose_origin"], out["compose_quat"] = _rows(compose, c["trafo_origin"], c["trafo_quat"], c["right_origin"],
                                                       c["right_quat"], out_shapes=[(3,), (4,)])
    return out


def pin_cases_reference(cases):
    """The reference's answers for the same cases, from oracle/_ref/librefpin.so.
    The push is BorisPusher::push between the unit switches of
    PartBunchBase.hpp:468-513 (R / (c dt) per component, then R * (c dt))."""
    L = reference_pin()
    if L is None:
        raise RuntimeError("oracle/_ref/librefpin.so is missing: the reference tree is needed")
    c = cases
    dt, mass, charge = (C.c_double(float(c[k])) for k in ("dt", "mass", "charge"))
    out = {}
    P = _f64(c["kick_P"]).copy()
    R0 = np.zeros(3)
    for i in range(len(P)):
        L.ref_boris_kick(_ptr(R0), _ptr(P[i]), _ptr(_f64(c["kick_Ef"][i])), _ptr(_f64(c["kick_Bf"][i])), dt, mass,
                         charge)
    out["kick"] = P
    R = _f64(c["push_R"]).copy()
    s = c_light() * float(c["dt"])
    for i in range(len(R)):
        r = np.array([R[i, 0] / s, R[i, 1] / s, R[i, 2] / s])
        L.ref_boris_push_unitless(_ptr(r), _ptr(_f64(c["push_P"][i])), dt)
        R[i] = [r[0] * s, r[1] * s, r[2] * s]
    out["push"] = R
    out["quaternion"], = _rows(L.ref_get_quaternion, c["quat_u"], c["quat_ref"], out_shapes=[(4,)])
    out["rotation_matrix"], = _rows(L.ref_rotation_matrix, c["rotmat_quat"], out_shapes=[(9,)])
    out["quaternion_rotate"], = _rows(L.ref_quaternion_rotate, c["trafo_quat"], c["trafo_r"], out_shapes=[(3,)])
    out["transform_to"], = _rows(L.ref_trafo_transform_to, c["trafo_origin"], c["trafo_quat"], c["trafo_r"],
                                 out_shapes=[(3,)])
    out["rotate_to"], = _rows(L.ref_trafo_rotate_to, c["trafo_origin"], c["trafo_quat"], c["trafo_r"],
                              out_shapes=[(3,)])
    out["inverted_origin"], out["inverted_quat"] = _rows(L.ref_trafo_inverted, c["trafo_origin"], c["trafo_quat"],
                                                         out_shapes=[(3,), (4,)])
    out["compose_origin"], out["compose_quat"] = _rows(L.ref_trafo_compose, c["trafo_origin"], c["trafo_quat"],
                                                       c["right_origin"], c["right_quat"], out_shapes=[(3,), (4,)])
    return out
