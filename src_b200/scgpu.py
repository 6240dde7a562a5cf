"""ctypes binding of the C ABI in include/scgpu.h (libscgpu.so, sm_100a).

The names follow the reference's call surface: ``FFTPoissonSolver``
(PoissonSolver::computePotential), ``PartBunch`` (computeSelfFields,
calcBeamParameters) and ``ParallelTTracker`` (the step loop).  There is no
CPU fallback: importing works anywhere, but creating a solver needs the
built library and a CUDA device, and fails loudly otherwise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libscgpu.so")

PLAIN_FP64 = 0
MIXED = 1
NSTATS = 28
FIELD_RHO, FIELD_PHI, FIELD_E = 0, 1, 2

ERRORS = {
    -1: "SCGPU_ERR_ARG", -2: "SCGPU_ERR_OOM", -3: "SCGPU_ERR_MESH", -4: "SCGPU_ERR_GUARD",
    -5: "SCGPU_ERR_FRAME", -6: "SCGPU_ERR_CUDA", -7: "SCGPU_ERR_STATE", -8: "SCGPU_ERR_UNSUPPORTED",
    -9: "SCGPU_ERR_EXCHANGE",
}

_dp = C.POINTER(C.c_double)
# scgpu_exchange_fn(device_buffer, count, op, cuda_stream, user) -> status
EXCHANGE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_longlong, C.c_int, C.c_void_p, C.c_void_p)


class SolverParams(C.Structure):
    _fields_ = [("mx", C.c_int), ("my", C.c_int), ("mt", C.c_int), ("precision", C.c_int), ("bboxincr", C.c_double)]


class BunchParams(C.Structure):
    _fields_ = [("dT", C.c_double), ("mass", C.c_double), ("charge", C.c_double), ("q_macro", C.c_double),
                ("coupling", C.c_double), ("bz_ext", C.c_double), ("t", C.c_double), ("path_length", C.c_double),
                ("ref_R", C.c_double * 3), ("ref_P", C.c_double * 3)]


class TrackerState(C.Structure):
    _fields_ = [("t", C.c_double), ("path_length", C.c_double), ("ref_R", C.c_double * 3), ("ref_P", C.c_double * 3),
                ("q_macro", C.c_double), ("ref_to_lab_origin", C.c_double * 3), ("ref_to_lab_quat", C.c_double * 4),
                ("step", C.c_longlong)]


class BeamParams(C.Structure):
    _fields_ = [(name, C.c_double * 3) for name in ("rmean", "pmean", "rrms", "prms", "eps_norm", "eps", "rprms")] + \
               [("gamma", C.c_double), ("moments", C.c_double * 27)]

    def as_dict(self):
        out = {name: np.array(getattr(self, name)) for name, _ in self._fields_ if name != "gamma"}
        out["gamma"] = float(self.gamma)
        return out


class Mesh(C.Structure):
    _fields_ = [("hr", C.c_double * 3), ("origin", C.c_double * 3), ("rmin", C.c_double * 3),
                ("rmax", C.c_double * 3), ("gammaz", C.c_double), ("hr_scaled", C.c_double * 3)]


class ScgpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def lib():
    """Load libscgpu.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C src_b200/csrc` "
                               "(or __graft_entry__.build()); there is no CPU fallback")
        L = C.CDLL(LIB_PATH)
        L.scgpu_last_error.restype = C.c_char_p
        L.scgpu_last_track_ms.restype = C.c_double
        L.scgpu_create.argtypes = [C.POINTER(C.c_void_p), C.POINTER(SolverParams), C.c_int]
        for name in ("scgpu_destroy", "scgpu_last_error", "scgpu_synchronize", "scgpu_last_track_ms"):
            getattr(L, name).argtypes = [C.c_void_p]
        L.scgpu_set_stream.argtypes = [C.c_void_p, C.c_void_p]
        L.scgpu_compute_potential.argtypes = [C.c_void_p, _dp, _dp]
        L.scgpu_compute_potential_device.argtypes = [C.c_void_p, C.c_void_p, _dp]
        L.scgpu_compute_self_fields.argtypes = [C.c_void_p, C.c_longlong, _dp, _dp, _dp, C.c_double, _dp, _dp]
        L.scgpu_register_host.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong]
        L.scgpu_unregister_host.argtypes = [C.c_void_p, C.c_void_p]
        L.scgpu_bunch_upload.argtypes = [C.c_void_p, C.c_longlong, _dp, _dp, C.POINTER(BunchParams)]
        L.scgpu_bunch_download.argtypes = [C.c_void_p, _dp, _dp]
        L.scgpu_track.argtypes = [C.c_void_p, C.c_int, _dp]
        L.scgpu_get_tracker_state.argtypes = [C.c_void_p, C.POINTER(TrackerState)]
        L.scgpu_beam_parameters.argtypes = [C.c_void_p, C.POINTER(BeamParams)]
        L.scgpu_beam_parameters_from_stats.argtypes = [_dp, C.c_longlong, C.POINTER(BeamParams)]
        L.scgpu_get_field.argtypes = [C.c_void_p, C.c_int, _dp]
        L.scgpu_get_mesh.argtypes = [C.c_void_p, C.POINTER(Mesh)]
        L.scgpu_profile_track.argtypes = [C.c_void_p, C.c_int, _dp]
        L.scgpu_kernels_per_step.argtypes = [C.c_void_p]
        _ip = C.POINTER(C.c_int)
        L.scgpu_compute_potential_image.argtypes = [C.c_void_p, _dp, _dp, C.c_double]
        L.scgpu_compute_potential_image_device.argtypes = [C.c_void_p, C.c_void_p, _dp, C.c_double]
        L.scgpu_compute_self_fields_binned.argtypes = [C.c_void_p, C.c_longlong, _dp, _dp, _ip, C.c_int, C.c_int,
                                                       C.c_double, C.c_double, _dp, _dp, _dp]
        L.scgpu_set_energy_bins.argtypes = [C.c_void_p, _ip, C.c_int, C.c_int]
        L.scgpu_get_bin_gammas.argtypes = [C.c_void_p, _dp, C.POINTER(C.c_longlong)]
        L.scgpu_set_periodic_z.argtypes = [C.c_void_p, C.c_int]
        L.scgpu_set_beam_frequency.argtypes = [C.c_void_p, C.c_double]
        L.scgpu_set_reorder_interval.argtypes = [C.c_void_p, C.c_int]
        L.scgpu_launch_count.argtypes = [C.c_void_p, C.POINTER(C.c_longlong)]
        L.scgpu_set_exchange.argtypes = [C.c_void_p, EXCHANGE_FN, C.c_void_p, C.c_longlong, C.c_int]
        L.scgpu_add_solenoid.argtypes = [C.c_void_p, C.c_char_p, C.c_double, C.c_double]
        L.scgpu_clear_elements.argtypes = [C.c_void_p]
        L.scgpu_fieldmap_astra1d.argtypes = [C.c_char_p, _dp, C.c_int, C.POINTER(C.c_int), _dp, _dp, _dp]
        L.scgpu_add_rfcavity.argtypes = [C.c_void_p, C.c_char_p, C.c_double, C.c_double, C.c_double, C.c_double]
        L.scgpu_fieldmap_2d.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), _dp,
                                        _dp, _dp, C.c_longlong]
        L.scgpu_fieldmap_3d.argtypes = [C.c_char_p, C.POINTER(C.c_int), _dp, _dp, _dp, C.c_longlong]
        L.scgpu_add_multipole.argtypes = [C.c_void_p, C.c_double, C.c_double, _dp, C.c_int, _dp, _dp, C.c_int, _dp]
        L.scgpu_fieldmap_astra1d_dynamic.argtypes = [C.c_char_p, _dp, C.c_int, C.POINTER(C.c_int), _dp, _dp, _dp, _dp]
        L.scgpu_stat_row.argtypes = [C.c_void_p, _dp]
        L.scgpu_stat_column_name.argtypes = [C.c_int]
        L.scgpu_stat_column_name.restype = C.c_char_p
        L.scgpu_sdds_write_header.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_char_p, C.c_char_p]
        L.scgpu_sdds_append_row.argtypes = [C.c_char_p, _dp, C.c_int]
        L.scgpu_read_fromfile_count.argtypes = [C.c_char_p, C.POINTER(C.c_longlong)]
        L.scgpu_read_fromfile.argtypes = [C.c_char_p, C.c_longlong, _dp, _dp, C.c_int, C.c_double,
                                          C.POINTER(C.c_longlong)]
        L.scgpu_write_fromfile.argtypes = [C.c_char_p, C.c_longlong, _dp, _dp]
        _lib = L
    return _lib


EXPORTED = [
    "scgpu_abi_version", "scgpu_create", "scgpu_destroy", "scgpu_last_error", "scgpu_set_stream",
    "scgpu_synchronize", "scgpu_compute_potential", "scgpu_compute_potential_device",
    "scgpu_compute_self_fields", "scgpu_register_host", "scgpu_unregister_host", "scgpu_bunch_upload",
    "scgpu_bunch_download", "scgpu_track", "scgpu_get_tracker_state", "scgpu_beam_parameters",
    "scgpu_beam_parameters_from_stats", "scgpu_get_field", "scgpu_get_mesh", "scgpu_last_track_ms",
    "scgpu_profile_track", "scgpu_kernels_per_step", "scgpu_compute_potential_image",
    "scgpu_compute_potential_image_device", "scgpu_compute_self_fields_binned", "scgpu_set_energy_bins",
    "scgpu_get_bin_gammas", "scgpu_stat_row", "scgpu_stat_column_name", "scgpu_sdds_write_header",
    "scgpu_sdds_append_row", "scgpu_read_fromfile_count", "scgpu_read_fromfile", "scgpu_write_fromfile",
    "scgpu_set_periodic_z", "scgpu_set_exchange", "scgpu_add_solenoid", "scgpu_clear_elements",
    "scgpu_fieldmap_astra1d", "scgpu_add_rfcavity", "scgpu_fieldmap_astra1d_dynamic", "scgpu_set_reorder_interval",
    "scgpu_launch_count", "scgpu_set_beam_frequency", "scgpu_add_multipole", "scgpu_fieldmap_2d",
    "scgpu_fieldmap_3d",
]
STAT_COLUMNS = 48
MAX_BINS = 64

PHASES = ["drift_bounds", "deposit", "assemble_rho", "green", "convolution", "grad", "gather_kick_push", "reorder"]


def _p(a):
    return a.ctypes.data_as(_dp)


def _f64c(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None and a.shape != shape:
        raise ValueError(f"expected shape {shape}, got {a.shape}")
    return a


class Context:
    """One solver instance on one device (FieldSolver + FFTPoissonSolver)."""

    def __init__(self, nr, precision=PLAIN_FP64, bboxincr=2.0, device=0):
        self.nr = tuple(int(v) for v in nr)
        self.precision = precision
        sp = SolverParams(self.nr[0], self.nr[1], self.nr[2], precision, float(bboxincr))
        h = C.c_void_p()
        rc = lib().scgpu_create(C.byref(h), C.byref(sp), int(device))
        if rc != 0:
            raise ScgpuError(rc, f"scgpu_create(nr={self.nr}, precision={precision}) failed")
        self.h = h
        self.n = 0
        self.nbins = 0

    def _check(self, rc, what):
        if rc != 0:
            msg = lib().scgpu_last_error(self.h)
            raise ScgpuError(rc, f"{what}: {msg.decode() if msg else ''}")

    def close(self):
        if getattr(self, "h", None):
            lib().scgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- PoissonSolver::computePotential
    def compute_potential(self, rho, hr):
        """rho: array [nz, ny, nx] (x fastest).  Returns the convolution."""
        r = _f64c(rho).copy()
        assert r.shape == (self.nr[2], self.nr[1], self.nr[0])
        self._check(lib().scgpu_compute_potential(self.h, _p(r), (C.c_double * 3)(*hr)), "compute_potential")
        return r

    # ---- beamline elements (computeExternalFields)
    def add_solenoid(self, fieldmap, elemedge, ks):
        """SOLENOID with an ASTRA 1D magnetostatic map at ELEMEDGE [m], KS [T]."""
        self._check(lib().scgpu_add_solenoid(self.h, os.fsencode(fieldmap), float(elemedge), float(ks)), "add_solenoid")

    def add_rfcavity(self, fieldmap, elemedge, volt, freq_mhz, lag):
        """RFCAVITY with an ASTRA dynamic map at ELEMEDGE [m]: VOLT [MV/m], FREQ [MHz], LAG [rad]."""
        self._check(lib().scgpu_add_rfcavity(self.h, os.fsencode(fieldmap), float(elemedge), float(volt),
                                             float(freq_mhz), float(lag)), "add_rfcavity")

    def add_multipole(self, elemedge, length, kn=(), dkn=None, ks=(), dks=None):
        """MULTIPOLE at ELEMEDGE [m] of length L [m]: normal / skew strengths
        KN, KS (order 1 = dipole first) with optional errors DKN, DKS."""
        def arr(v, n):
            if v is None:
                return None
            a = np.ascontiguousarray(np.broadcast_to(np.asarray(v, dtype=np.float64), (n,)))
            return a
        kn_a, ks_a = arr(kn, len(kn)), arr(ks, len(ks))
        dkn_a, dks_a = arr(dkn, len(kn)), arr(dks, len(ks))
        p = lambda a: _p(a) if a is not None and a.size else None
        self._check(lib().scgpu_add_multipole(self.h, float(elemedge), float(length), p(kn_a), len(kn), p(dkn_a),
                                              p(ks_a), len(ks), p(dks_a)), "add_multipole")

    def clear_elements(self):
        self._check(lib().scgpu_clear_elements(self.h), "clear_elements")

    def launch_count(self):
        """Kernels scgpu_track has launched on this context so far."""
        n = C.c_longlong(0)
        self._check(lib().scgpu_launch_count(self.h, C.byref(n)), "launch_count")
        return int(n.value)

    def set_reorder_interval(self, steps):
        """Cell reorder every `steps` tracked steps (0: never); results do not change."""
        self._check(lib().scgpu_set_reorder_interval(self.h, int(steps)), "set_reorder_interval")

    # ---- FIELDSOLVER BCFFTZ=PERIODIC: periodic-z solves and a DC beam
    def set_periodic_z(self, periodic=True):
        """Cyclic convolution along z; the tracked bunch becomes a DC beam
        (the period's mesh along z, the periodic particle boundary)."""
        self._check(lib().scgpu_set_periodic_z(self.h, 1 if periodic else 0), "set_periodic_z")

    def set_beam_frequency(self, f_hz):
        """setBeamFrequency: the DC beam's period length c / f."""
        self._check(lib().scgpu_set_beam_frequency(self.h, float(f_hz)), "set_beam_frequency")

    # ---- PoissonSolver::computePotential(rho, hr, zshift): image charge
    def compute_potential_image(self, rho, hr, zshift):
        """rho: array [nz, ny, nx].  Returns the image charge's potential
        (minus the shifted convolution, z flipped)."""
        r = _f64c(rho).copy()
        assert r.shape == (self.nr[2], self.nr[1], self.nr[0])
        self._check(lib().scgpu_compute_potential_image(self.h, _p(r), (C.c_double * 3)(*hr), float(zshift)),
                    "compute_potential_image")
        return r

    # ---- the energy-bin loop of computeSpaceChargeFields
    def compute_self_fields_binned(self, R, P, bins, nbins, q_macro, dT, last_emitted=None):
        """Beam-frame bunch with one energy bin per particle.  Returns Ef, Bf
        (summed over the emitted bins and their images) and the bin gammas."""
        R = _f64c(R)
        P = _f64c(P)
        n = R.shape[0]
        b = np.ascontiguousarray(bins, dtype=np.int32)
        assert b.shape == (n,)
        Ef = np.empty_like(R)
        Bf = np.empty_like(R)
        g = np.empty(max(int(nbins), 1))
        le = int(nbins) if last_emitted is None else int(last_emitted)
        self._check(lib().scgpu_compute_self_fields_binned(self.h, n, _p(R), _p(P), b.ctypes.data_as(C.POINTER(C.c_int)),
                                                           int(nbins), le, float(q_macro), float(dT), _p(Ef), _p(Bf),
                                                           _p(g)), "compute_self_fields_binned")
        return Ef, Bf, g[:int(nbins)]

    def set_energy_bins(self, bins, nbins, last_emitted=None):
        """Energy bins of the resident bunch (order of the last upload);
        nbins = 0 returns to one self-field solve."""
        le = int(nbins) if last_emitted is None else int(last_emitted)
        if int(nbins) == 0:
            self._check(lib().scgpu_set_energy_bins(self.h, None, 0, le), "set_energy_bins")
            return
        b = np.ascontiguousarray(bins, dtype=np.int32)
        if self.n and b.shape != (self.n,):
            raise ValueError(f"bins: expected shape ({self.n},), got {b.shape}")
        self._check(lib().scgpu_set_energy_bins(self.h, b.ctypes.data_as(C.POINTER(C.c_int)), int(nbins), le),
                    "set_energy_bins")
        self.nbins = int(nbins)

    def stat_row(self):
        """One row of the reference's .stat file for the resident bunch."""
        row = np.empty(STAT_COLUMNS)
        self._check(lib().scgpu_stat_row(self.h, _p(row)), "stat_row")
        return row

    def bin_gammas(self):
        g = np.empty(self.nbins)
        cnt = np.empty(self.nbins, dtype=np.int64)
        self._check(lib().scgpu_get_bin_gammas(self.h, _p(g), cnt.ctypes.data_as(C.POINTER(C.c_longlong))),
                    "get_bin_gammas")
        return g, cnt

    # ---- PartBunch::computeSelfFields
    def compute_self_fields(self, R, P, q_macro, dT):
        R = _f64c(R)
        P = _f64c(P)
        n = R.shape[0]
        Ef = np.empty_like(R)
        Bf = np.empty_like(R)
        q = C.c_double(q_macro)
        self._check(lib().scgpu_compute_self_fields(self.h, n, _p(R), _p(P), C.byref(q), float(dT), _p(Ef), _p(Bf)),
                    "compute_self_fields")
        return Ef, Bf, q.value

    # ---- bunch state
    def upload(self, R, P, dT, q_macro, mass, charge=-1.0, coupling=None, bz_ext=0.0, t=0.0, path_length=0.0,
               ref_R=(0.0, 0.0, 0.0), ref_P=(0.0, 0.0, 10.0)):
        R = _f64c(R)
        P = _f64c(P)
        if coupling is None:
            coupling = 1.0 / (4 * 3.14159265358979323846 * 8.854187817e-12)
        bp = BunchParams(dT, mass, charge, q_macro, coupling, bz_ext, t, path_length, (C.c_double * 3)(*ref_R),
                         (C.c_double * 3)(*ref_P))
        self._check(lib().scgpu_bunch_upload(self.h, R.shape[0], _p(R), _p(P), C.byref(bp)), "bunch_upload")
        self.n = R.shape[0]
        self.nbins = 0

    def download(self, R=None, P=None):
        """Returns R, P (n x 3); pass pinned arrays to receive them in place."""
        R = np.empty((self.n, 3)) if R is None else R
        P = np.empty((self.n, 3)) if P is None else P
        assert R.dtype == np.float64 and R.flags.c_contiguous and R.shape == (self.n, 3)
        assert P.dtype == np.float64 and P.flags.c_contiguous and P.shape == (self.n, 3)
        self._check(lib().scgpu_bunch_download(self.h, _p(R), _p(P)), "bunch_download")
        return R, P

    def track(self, nsteps, stats=None):
        """stats: optional float64 array [nsteps, NSTATS] (pinned for best overlap)."""
        sp = None
        if stats is not None:
            assert stats.dtype == np.float64 and stats.flags.c_contiguous and stats.size >= nsteps * NSTATS
            sp = _p(stats)
        self._check(lib().scgpu_track(self.h, int(nsteps), sp), "track")
        return lib().scgpu_last_track_ms(self.h)

    def tracker_state(self):
        s = TrackerState()
        self._check(lib().scgpu_get_tracker_state(self.h, C.byref(s)), "get_tracker_state")
        return {"t": s.t, "path_length": s.path_length, "ref_R": np.array(s.ref_R), "ref_P": np.array(s.ref_P),
                "q_macro": s.q_macro, "step": s.step, "ref_to_lab_origin": np.array(s.ref_to_lab_origin),
                "ref_to_lab_quat": np.array(s.ref_to_lab_quat)}

    def beam_parameters(self):
        bp = BeamParams()
        self._check(lib().scgpu_beam_parameters(self.h, C.byref(bp)), "beam_parameters")
        return bp.as_dict()

    def field(self, which):
        nx, ny, nz = self.nr
        out = np.empty((nz, ny, nx, 3) if which == FIELD_E else (nz, ny, nx))
        self._check(lib().scgpu_get_field(self.h, which, _p(out)), "get_field")
        return out

    def profile(self, nsteps):
        """Per-phase device milliseconds summed over nsteps serialised steps."""
        out = np.zeros(len(PHASES))
        self._check(lib().scgpu_profile_track(self.h, int(nsteps), _p(out)), "profile_track")
        return dict(zip(PHASES, out))

    def kernels_per_step(self):
        k = lib().scgpu_kernels_per_step(self.h)
        if k < 0:
            self._check(k, "kernels_per_step")
        return k

    def set_stream(self, stream_handle):
        self._check(lib().scgpu_set_stream(self.h, C.c_void_p(stream_handle)), "set_stream")

    def mesh(self):
        m = Mesh()
        self._check(lib().scgpu_get_mesh(self.h, C.byref(m)), "get_mesh")
        return {"hr": np.array(m.hr), "origin": np.array(m.origin), "rmin": np.array(m.rmin),
                "rmax": np.array(m.rmax), "gammaz": m.gammaz, "hr_scaled": np.array(m.hr_scaled)}


def beam_parameters_from_stats(record, n):
    bp = BeamParams()
    rec = _f64c(record)
    rc = lib().scgpu_beam_parameters_from_stats(_p(rec), int(n), C.byref(bp))
    if rc != 0:
        raise ScgpuError(rc, "beam_parameters_from_stats")
    return bp.as_dict()


# ---------------------------------------------------------------- batches
def _batch_lib():
    L = lib()
    if not getattr(L, "_batch_ready", False):
        L.scgpu_batch_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int]
        L.scgpu_batch_destroy.argtypes = [C.c_void_p]
        L.scgpu_batch_last_error.argtypes = [C.c_void_p]
        L.scgpu_batch_last_error.restype = C.c_char_p
        L.scgpu_batch_add.argtypes = [C.c_void_p, C.POINTER(SolverParams), C.c_longlong, _dp, _dp,
                                      C.POINTER(BunchParams)]
        L.scgpu_batch_remove.argtypes = [C.c_void_p, C.c_int]
        L.scgpu_batch_member.argtypes = [C.c_void_p, C.c_int]
        L.scgpu_batch_member.restype = C.c_void_p
        L.scgpu_batch_size.argtypes = [C.c_void_p]
        L.scgpu_batch_track.argtypes = [C.c_void_p, C.c_int]
        L.scgpu_batch_last_track_ms.argtypes = [C.c_void_p]
        L.scgpu_batch_last_track_ms.restype = C.c_double
        L.scgpu_batch_set_tuning.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
        L.scgpu_batch_get_tuning.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.scgpu_batch_autotune.argtypes = [C.c_void_p, C.c_int]
        L.scgpu_batch_launch.argtypes = [C.c_void_p, C.c_int]
        L.scgpu_batch_wait.argtypes = [C.c_void_p]
        L.scgpu_batch_done.argtypes = [C.c_void_p]
        L.scgpu_batch_trim.argtypes = [C.c_void_p]
        L._batch_ready = True
    return L


EXPORTED += [
    "scgpu_compute_potential_noalloc",
    "scgpu_batch_create", "scgpu_batch_destroy", "scgpu_batch_last_error", "scgpu_batch_add", "scgpu_batch_remove",
    "scgpu_batch_member", "scgpu_batch_size", "scgpu_batch_track", "scgpu_batch_last_track_ms",
    "scgpu_batch_set_tuning", "scgpu_batch_get_tuning", "scgpu_batch_autotune", "scgpu_batch_launch",
    "scgpu_batch_wait", "scgpu_batch_trim", "scgpu_batch_done",
]


class _Member(Context):
    """A bunch of a Batch: the single-bunch calls on the batch's slot context
    (the batch owns the context; closing the view does nothing)."""

    def __init__(self, handle, nr, precision, n):
        self.h = C.c_void_p(handle)
        self.nr = tuple(nr)
        self.precision = precision
        self.n = n

    def close(self):
        self.h = None


def _bunch_params(dT, q_macro, mass, charge=-1.0, coupling=None, bz_ext=0.0, t=0.0, path_length=0.0,
                  ref_R=(0.0, 0.0, 0.0), ref_P=(0.0, 0.0, 10.0)):
    if coupling is None:
        coupling = 1.0 / (4 * 3.14159265358979323846 * 8.854187817e-12)
    return BunchParams(dT, mass, charge, q_macro, coupling, bz_ext, t, path_length, (C.c_double * 3)(*ref_R),
                       (C.c_double * 3)(*ref_P))


class Batch:
    """Many bunches stepping together (scgpu_batch_*): one launch per kernel
    of the step for all bunches, one graph launch per step."""

    def __init__(self, precision=PLAIN_FP64, device=0):
        h = C.c_void_p()
        rc = _batch_lib().scgpu_batch_create(C.byref(h), int(device), int(precision))
        if rc != 0:
            raise ScgpuError(rc, "scgpu_batch_create failed")
        self.h = h
        self.precision = precision
        self._meta = {}

    def _check(self, rc, what):
        if rc < 0:
            msg = _batch_lib().scgpu_batch_last_error(self.h)
            raise ScgpuError(rc, f"{what}: {msg.decode() if msg else ''}")
        return rc

    def close(self):
        if getattr(self, "h", None):
            _batch_lib().scgpu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add(self, nr, R, P, dT, q_macro, mass, bboxincr=2.0, **kw):
        """Uploads a bunch on a mesh nr = (mx, my, mt); returns its slot."""
        R = _f64c(R)
        P = _f64c(P)
        nr = tuple(int(v) for v in nr)
        sp = SolverParams(nr[0], nr[1], nr[2], self.precision, float(bboxincr))
        bp = _bunch_params(dT, q_macro, mass, **kw)
        slot = self._check(_batch_lib().scgpu_batch_add(self.h, C.byref(sp), R.shape[0], _p(R), _p(P), C.byref(bp)),
                           "batch_add")
        self._meta[slot] = (nr, R.shape[0])
        return slot

    def remove(self, slot):
        self._check(_batch_lib().scgpu_batch_remove(self.h, int(slot)), "batch_remove")
        self._meta.pop(slot, None)

    def member(self, slot):
        h = _batch_lib().scgpu_batch_member(self.h, int(slot))
        if not h:
            raise ScgpuError(-1, f"no bunch in slot {slot}")
        nr, n = self._meta[slot]
        return _Member(h, nr, self.precision, n)

    def size(self):
        return _batch_lib().scgpu_batch_size(self.h)

    def track(self, nsteps):
        self._check(_batch_lib().scgpu_batch_track(self.h, int(nsteps)), "batch_track")
        return _batch_lib().scgpu_batch_last_track_ms(self.h)

    def launch(self, nsteps):
        """Enqueues nsteps batched steps and returns at once; wait() ends them."""
        self._check(_batch_lib().scgpu_batch_launch(self.h, int(nsteps)), "batch_launch")

    def wait(self):
        """Finishes launched steps; returns their device milliseconds."""
        self._check(_batch_lib().scgpu_batch_wait(self.h), "batch_wait")
        return _batch_lib().scgpu_batch_last_track_ms(self.h)

    def done(self):
        """True when the launched steps have finished on the device (never blocks)."""
        rc = _batch_lib().scgpu_batch_done(self.h)
        if rc < 0:
            self._check(rc, "batch_done")
        return rc == 1

    def trim(self):
        """Frees the parked contexts of removed bunches."""
        self._check(_batch_lib().scgpu_batch_trim(self.h), "batch_trim")

    def set_tuning(self, deposit_threads=256, L=0, fft_variant=0):
        self._check(_batch_lib().scgpu_batch_set_tuning(self.h, int(deposit_threads), int(L), int(fft_variant)),
                    "batch_set_tuning")

    def tuning(self, L):
        t, v = C.c_int(), C.c_int()
        self._check(_batch_lib().scgpu_batch_get_tuning(self.h, int(L), C.byref(t), C.byref(v)), "batch_get_tuning")
        return {"deposit_threads": t.value, "fft_variant": v.value}

    def autotune(self, trial_steps=3):
        """Times the candidate launch shapes on the current bunches; returns
        the number of steps the trials advanced every bunch."""
        return self._check(_batch_lib().scgpu_batch_autotune(self.h, int(trial_steps)), "batch_autotune")


# ---- the reference's file formats (host side of the C ABI; no device needed)
def stat_column_names():
    return [lib().scgpu_stat_column_name(i).decode() for i in range(STAT_COLUMNS)]


class StatWriter:
    """DataSink's SDDS statistics file: the header on creation, one row per
    write(row) (rows from Context.stat_row)."""

    def __init__(self, path, input_name="", processors=1, revision="", flavor="opal-t", with_particle0=True):
        self.path = os.fsencode(path)
        self.with_particle0 = with_particle0
        rc = lib().scgpu_sdds_write_header(self.path, input_name.encode(), int(processors), revision.encode(),
                                           flavor.encode())
        if rc != 0:
            raise ScgpuError(rc, f"cannot write {path}")

    def write(self, row):
        r = _f64c(row, (STAT_COLUMNS,))
        rc = lib().scgpu_sdds_append_row(self.path, _p(r), 1 if self.with_particle0 else 0)
        if rc != 0:
            raise ScgpuError(rc, "cannot append a statistics row")


def read_fromfile(path, momenta_in_ev=False, mass_ev=0.51099892e6):
    """DISTRIBUTION TYPE=FROMFILE: returns R, P (n x 3, P as beta*gamma)."""
    n = C.c_longlong(0)
    rc = lib().scgpu_read_fromfile_count(os.fsencode(path), C.byref(n))
    if rc != 0:
        raise ScgpuError(rc, f"{path} does not hold an ASCII distribution")
    R = np.empty((n.value, 3))
    P = np.empty((n.value, 3))
    rc = lib().scgpu_read_fromfile(os.fsencode(path), n.value, _p(R), _p(P), 1 if momenta_in_ev else 0,
                                   float(mass_ev), C.byref(n))
    if rc != 0:
        raise ScgpuError(rc, f"cannot read {path}")
    return R, P


def write_fromfile(path, R, P):
    R = _f64c(R)
    P = _f64c(P)
    rc = lib().scgpu_write_fromfile(os.fsencode(path), R.shape[0], _p(R), _p(P))
    if rc != 0:
        raise ScgpuError(rc, f"cannot write {path}")


def fieldmap_astra1d(path):
    """Astra1DMagnetoStatic::readMap: (Fourier coefficients, zbegin, zend, period)."""
    coefs = np.empty(255)
    n = C.c_int(0)
    zb, ze, per = C.c_double(), C.c_double(), C.c_double()
    rc = lib().scgpu_fieldmap_astra1d(os.fsencode(path), _p(coefs), 255, C.byref(n), C.byref(zb), C.byref(ze),
                                      C.byref(per))
    if rc != 0:
        raise ScgpuError(rc, f"cannot read the field map {path}")
    return coefs[:n.value].copy(), zb.value, ze.value, per.value


def fieldmap_2d(path):
    """A 2D (r, z) map as the library reads it: dict with dynamic, nz, nr,
    zbegin, zend, rbegin, rend [m], freq_mhz and values [component, r, z]."""
    dyn, nz, nr = C.c_int(), C.c_int(), C.c_int()
    ranges = (C.c_double * 4)()
    f = C.c_double()
    rc = lib().scgpu_fieldmap_2d(os.fsencode(path), C.byref(dyn), C.byref(nz), C.byref(nr), ranges, C.byref(f), None, 0)
    if rc:
        raise ScgpuError(rc, f"fieldmap_2d: cannot read {path}")
    nc = 3 if dyn.value else 2
    v = np.empty((nc, nr.value, nz.value))
    rc = lib().scgpu_fieldmap_2d(os.fsencode(path), C.byref(dyn), C.byref(nz), C.byref(nr), ranges, C.byref(f),
                                 _p(v), v.size)
    if rc:
        raise ScgpuError(rc, f"fieldmap_2d: cannot read {path}")
    return dict(dynamic=bool(dyn.value), nz=nz.value, nr=nr.value, zbegin=ranges[0], zend=ranges[1], rbegin=ranges[2],
                rend=ranges[3], freq_mhz=f.value, values=v)


def fieldmap_3d(path):
    """A 3D dynamic map as the library reads it: dict with nx, ny, nz (grid
    points), xbegin, xend, ybegin, yend, zbegin, zend [m], freq_mhz and values
    [component, x, y, z] (Ex, Ey, Ez [V/m], Bx, By, Bz [T])."""
    n = (C.c_int * 3)()
    ranges = (C.c_double * 6)()
    f = C.c_double()
    rc = lib().scgpu_fieldmap_3d(os.fsencode(path), n, ranges, C.byref(f), None, 0)
    if rc:
        raise ScgpuError(rc, f"fieldmap_3d: cannot read {path}")
    v = np.empty((6, n[0], n[1], n[2]))
    rc = lib().scgpu_fieldmap_3d(os.fsencode(path), n, ranges, C.byref(f), _p(v), v.size)
    if rc:
        raise ScgpuError(rc, f"fieldmap_3d: cannot read {path}")
    keys = ("xbegin", "xend", "ybegin", "yend", "zbegin", "zend")
    return dict(nx=n[0], ny=n[1], nz=n[2], freq_mhz=f.value, values=v, **{k: ranges[i] for i, k in enumerate(keys)})


def fieldmap_astra1d_dynamic(path):
    """Astra1DDynamic::readMap: (coefficients in V/m per MV/m, zbegin, zend, period, frequency [MHz])."""
    coefs = np.empty(255)
    n = C.c_int(0)
    zb, ze, per, f = C.c_double(), C.c_double(), C.c_double(), C.c_double()
    rc = lib().scgpu_fieldmap_astra1d_dynamic(os.fsencode(path), _p(coefs), 255, C.byref(n), C.byref(zb), C.byref(ze),
                                              C.byref(per), C.byref(f))
    if rc != 0:
        raise ScgpuError(rc, f"cannot read the field map {path}")
    return coefs[:n.value].copy(), zb.value, ze.value, per.value, f.value