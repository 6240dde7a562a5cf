"""CPU tests of the drop-in boundary: libscgpu.so loads, exports every entry
point that include/scgpu.h declares, and validates its arguments before it
touches a device (no compute calls here)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from src_b200 import scgpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for hdr in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not hdr.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", hdr)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(scgpu_[a-z0-9_]+)\s*\(", text))
    return names


def test_header_declares_the_python_binding():
    assert set(scgpu.EXPORTED) <= declared_symbols()


def test_library_exports_every_declared_symbol():
    L = scgpu.lib()
    missing = [n for n in sorted(declared_symbols()) if not hasattr(L, n)]
    assert not missing, missing


def test_abi_version():
    assert scgpu.lib().scgpu_abi_version() == 1


@pytest.mark.parametrize("mx,my,mt,prec,bbox,code", [
    (64, 64, 64, 7, 2.0, -1),      # unknown precision
    (2, 64, 64, 0, 2.0, -8),       # Grad needs 3 cells
    (64, 64, 200, 0, 2.0, -8),     # doubled length above 256
    (7, 64, 64, 0, 2.0, -8),       # 14 has the factor 7
    (64, 64, 64, 0, -1.0, -1),     # negative BBOXINCR
])
def test_create_rejects_bad_parameters_without_a_device(mx, my, mt, prec, bbox, code):
    sp = scgpu.SolverParams(mx, my, mt, prec, bbox)
    h = C.c_void_p()
    assert scgpu.lib().scgpu_create(C.byref(h), C.byref(sp), 0) == code
    assert not h.value


def test_null_arguments_are_rejected():
    L = scgpu.lib()
    assert L.scgpu_create(None, None, 0) == -1
    assert L.scgpu_set_stream(None, None) == -1
    assert L.scgpu_track(None, 1, None) == -1
    assert L.scgpu_set_reorder_interval(None, 8) == -1
    assert L.scgpu_launch_count(None, None) == -1
    out = scgpu.BeamParams()
    assert L.scgpu_beam_parameters_from_stats(None, 10, C.byref(out)) == -1


def test_beam_parameters_from_stats_matches_oracle(oracle):
    """Host-side calcBeamParameters of the C ABI against the oracle's."""
    from src_b200.bunch import gaussian_bunch
    R, P = gaussian_bunch(4000, bunch_id=21)
    bo = oracle.beam_parameters(R, P)
    rec = np.concatenate([bo["moments"], [oracle.lib().sco_sum_gamma(C.c_longlong(4000),
                                                                      P.ctypes.data_as(C.POINTER(C.c_double)))]])
    bg = scgpu.beam_parameters_from_stats(rec, 4000)
    for k in ("rmean", "pmean", "rrms", "prms", "eps_norm", "eps", "rprms"):
        np.testing.assert_array_equal(bg[k], bo[k])
    assert bg["gamma"] == bo["gamma"]


def test_bunch_generator_is_seeded():
    from src_b200.bunch import gaussian_bunch
    a = gaussian_bunch(1000, bunch_id=3)
    b = gaussian_bunch(1000, bunch_id=3)
    c = gaussian_bunch(1000, bunch_id=4)
    np.testing.assert_array_equal(a[0], b[0])
    assert not np.array_equal(a[0], c[0])
