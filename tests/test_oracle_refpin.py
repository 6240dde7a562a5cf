"""The oracle's frame and pusher arithmetic pinned to the reference's own
code: src/Steppers/BorisPusher.h (kick, push), src/Classic/Algorithms/
Quaternion.cpp (getQuaternion, getRotationMatrix, rotate) and
src/Classic/Algorithms/CoordinateSystemTrafo.{h,cpp} (transformTo, rotateTo,
inverted, operator*), compiled from the reference's sources by
oracle/Makefile into oracle/_ref/librefpin.so.

Both sides must give the same doubles, bit for bit, on every case:
* against tests/golden/refpin_kat.npz (the reference's answers, written by
  tests/golden/make_golden.py), everywhere;
* against the live reference library when the reference tree was there to
  build it.

The push is BorisPusher::push between the unit switches of
PartBunchBase.hpp:468-513 (R / (c dt), push, R * (c dt)), as the tracker
calls it.  The GPU parity tests compare the device with this oracle.
"""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "refpin_kat.npz")
KEYS = ("kick", "push", "quaternion", "rotation_matrix", "quaternion_rotate", "transform_to", "rotate_to",
        "inverted_origin", "inverted_quat", "compose_origin", "compose_quat")


def _cases():
    g = np.load(GOLD)
    return {k[3:]: g[k] for k in g.files if k.startswith("in_")}, {k[4:]: g[k] for k in g.files if k.startswith("ref_")}


def test_oracle_equals_reference_golden(oracle):
    cases, ref = _cases()
    got = oracle.pin_cases_oracle(cases)
    for k in KEYS:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)


def test_oracle_equals_live_reference(oracle):
    if not oracle.reference_pin_available():
        pytest.skip("oracle/_ref/librefpin.so not built (no reference tree on this machine)")
    cases, golden = _cases()
    live = oracle.pin_cases_reference(cases)
    got = oracle.pin_cases_oracle(cases)
    for k in KEYS:
        np.testing.assert_array_equal(live[k], golden[k], err_msg=k)
        np.testing.assert_array_equal(got[k], live[k], err_msg=k)


def test_pinning_cases_cover_the_branches(oracle):
    """The cases reach getQuaternion's parallel branch (identity) and its
    general branch, and kicks with and without a magnetic field."""
    cases, ref = _cases()
    q = ref["quaternion"]
    ident = np.all(q == np.array([1.0, 0.0, 0.0, 0.0]), axis=1)
    assert 0 < ident.sum() < len(q)
    assert np.any(np.all(cases["kick_Bf"] == 0.0, axis=1)) and np.any(np.any(cases["kick_Bf"] != 0.0, axis=1))
