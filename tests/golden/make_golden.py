"""Generate the golden fixtures in tests/golden/ (run in a tree that has the
reference sources, after `make -C oracle`).

fftpack_kat.npz
    Inputs and outputs of the reference's own FFTPACK (ippl/src/FFT/fftpack.cpp,
    compiled from source into oracle/_ref/libfftpack_ref.so): cfftf, cfftb,
    rfftf, rfftb at the doubled-grid lengths of the supported meshes.  The
    oracle's project-written FFT engine is checked against these.
convolution_n8.npz
    rho, hr and the open-boundary convolution of FFTPoissonSolver::computePotential
    computed by the oracle with the reference's FFTPACK engine, plus the
    mirrored integrated Green's function G2 (n = 8, non-cubic spacing).
step_n8.npz
    A 2000-particle bunch tracked 3 steps on an 8^3 mesh by the oracle with the
    reference's FFTPACK engine: final R, P and the last step's rho, phi, E.
image_n8.npz
    rho, hr, zshift and the image-charge potential of
    FFTPoissonSolver::computePotential(rho, hr, zshift) with the shifted
    Green's function G2s, by the oracle with the reference's FFTPACK engine.
binned_step_n8.npz
    A 3000-particle photoinjector bunch with 4 energy bins tracked 3 steps by
    the energy-bin loop with image charges (oracle, reference FFTPACK): final
    R, P and the last step's Ef, Bf.
refpin_kat.npz
    Random inputs and the answers of the reference's own BorisPusher::kick /
    push, getQuaternion, Quaternion::getRotationMatrix / rotate and
    CoordinateSystemTrafo::transformTo / rotateTo / inverted / operator*,
    compiled from src/ into oracle/_ref/librefpin.so (``python
    tests/golden/make_golden.py refpin`` writes only this file).
sdds_stat_columns.json
    The column definitions (name, type, units, description), the &data block
    and the parameter rows of the reference's SDDS statistics file, read from
    src/Structure/DataSink.cpp (writeSDDSHeader).

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from src_b200.bunch import gaussian_bunch  # noqa: E402

LENGTHS = (16, 32, 48, 64, 96, 128, 256)


def main():
    O.build()
    if not O.reference_fft_available():
        raise SystemExit("oracle/_ref/libfftpack_ref.so is missing: the reference tree is needed")
    O.use_reference_fft(True)
    rng = np.random.default_rng(20261203)
    kat = {}
    for n in LENGTHS:
        c = rng.standard_normal(2 * n)
        r = rng.standard_normal(n)
        kat[f"c_in_{n}"] = c
        kat[f"r_in_{n}"] = r
        kat[f"cfftf_{n}"] = O.fft1d(0, c)
        kat[f"cfftb_{n}"] = O.fft1d(1, c)
        kat[f"rfftf_{n}"] = O.fft1d(2, r)
        kat[f"rfftb_{n}"] = O.fft1d(3, r)
    np.savez_compressed(os.path.join(HERE, "fftpack_kat.npz"), **kat)

    nr = (8, 8, 8)
    hr = (2.5e-4, 3.0e-4, 4.0e-3)
    rho = rng.standard_normal((nr[2], nr[1], nr[0]))
    phi = O.compute_potential(rho, hr)
    G2 = O.igf(nr, hr)
    np.savez_compressed(os.path.join(HERE, "convolution_n8.npz"), rho=rho, hr=np.array(hr), phi=phi, G2=G2)

    R, P = gaussian_bunch(2000, bunch_id=7)
    R0, P0 = R.copy(), P.copy()
    prm = O.make_params(nr, 1e-12)
    tr = O.OracleTracker(prm, -1e-9 / 2000)
    dbg = tr.track(R, P, 3, want_debug=True)
    np.savez_compressed(os.path.join(HERE, "step_n8.npz"), R0=R0, P0=P0, R=R, P=P, rho=dbg["rho"], phi=dbg["phi"],
                        E=dbg["E"], Q=tr.Q, path_length=tr.path_length, t=tr.t)
    image_and_bins()
    sdds_columns()
    O.use_reference_fft(False)
    print("wrote fftpack_kat.npz, convolution_n8.npz, step_n8.npz, image_n8.npz, binned_step_n8.npz")


def image_and_bins():
    from src_b200.bunch import photoinjector_bunch  # noqa: E402
    rng = np.random.default_rng(20261205)
    nr = (8, 8, 8)
    hr = (2.5e-4, 3.0e-4, 4.0e-3)
    zshift = -3.3e-2
    rho = rng.standard_normal((nr[2], nr[1], nr[0]))
    phi = O.compute_potential_shifted(rho, hr, zshift)
    G2s = O.igf_shifted(nr, hr, zshift)
    np.savez_compressed(os.path.join(HERE, "image_n8.npz"), rho=rho, hr=np.array(hr), zshift=zshift, phi=phi, G2s=G2s)
    R, P, bins = photoinjector_bunch(3000, nbins=4, bunch_id=9)
    R0, P0 = R.copy(), P.copy()
    tr = O.OracleTracker(O.make_params(nr, 1e-12, ref_pz=1.0), -1e-9 / 3000)
    dbg = tr.track(R, P, 3, want_debug=True, bins=bins, nbins=4)
    np.savez_compressed(os.path.join(HERE, "binned_step_n8.npz"), R0=R0, P0=P0, bins=bins, R=R, P=P, Ef=dbg["Ef"],
                        Bf=dbg["Bf"], Q=tr.Q)


def sdds_columns():
    import json
    import re
    ref = os.environ.get("REF_DIR", "/root/reference")
    src = open(os.path.join(ref, "src", "Structure", "DataSink.cpp")).read()
    i = src.index("void DataSink::writeSDDSHeader(std::ofstream &outputFile,\n")
    j = src.index("void DataSink::", i + 50)
    blk = src[i:j]
    cols = re.findall(r'&column\\n"\s*<< indent << "name=([^,]*),\\n"\s*<< indent << "type=([^,]*),\\n"'
                      r'\s*<< indent << "units=([^,]*),\\n"\s*<< indent << "description=\\"([^"]*)\\"', blk)
    params = re.findall(r'&parameter\\n"\s*<< indent << "name=([^,]*),\\n"\s*<< indent << "type=([^,]*),', blk)
    data = re.findall(r'<< indent << "(mode=ascii,|no_row_counts=1)', blk)
    out = {"source": "src/Structure/DataSink.cpp writeSDDSHeader", "columns": cols, "parameters": params,
           "data": data, "value_format": "scientific, precision 15 (DataSink::open_m), then setw(10) << tab"}
    with open(os.path.join(HERE, "sdds_stat_columns.json"), "w") as f:
        json.dump(out, f, indent=1)


def pin_cases(seed=20261204):
    """Random inputs of the pinning cases: Boris kicks and pushes of beam-like
    and arbitrary momenta, getQuaternion of mean momenta near the z axis and
    of arbitrary directions, trafos with random origins and
    orientations, rotation matrices of not quite normalised quaternions."""
    rng = np.random.default_rng(seed)
    n = 1000
    c = {"dt": 1e-12, "mass": O.electron_mass_ev(), "charge": -1.0}
    beam = np.column_stack([1e-3 * rng.standard_normal(n), 1e-3 * rng.standard_normal(n),
                            10.0 * (1 + 1e-3 * rng.standard_normal(n))])
    anyp = rng.standard_normal((n, 3)) * np.exp(rng.uniform(np.log(0.05), np.log(50.0), (n, 1)))
    c["kick_P"] = np.concatenate([beam, anyp])
    c["kick_Ef"] = rng.standard_normal((2 * n, 3)) * np.exp(rng.uniform(np.log(1e3), np.log(1e8), (2 * n, 1)))
    Bf = 0.3 * rng.standard_normal((2 * n, 3))
    Bf[: n // 4] = 0.0
    c["kick_Bf"] = Bf
    c["push_R"] = 1e-3 * rng.standard_normal((2 * n, 3))
    c["push_P"] = c["kick_P"].copy()
    near = np.column_stack([1e-6 * rng.standard_normal(n), 1e-6 * rng.standard_normal(n),
                            10.0 * (1 + 1e-3 * rng.standard_normal(n))])
    near[: n // 8, :2] *= 1e-8   # within getQuaternion's parallel tolerance
    u_any = rng.standard_normal((n, 3))
    ref_any = rng.standard_normal((n, 3))
    flip = np.sum(u_any * ref_any, axis=1) < 0
    u_any[flip] *= -1.0          # no anti-parallel pairs (the reference draws a random axis there)
    zhat = np.tile([0.0, 0.0, 1.0], (n, 1))
    c["quat_u"] = np.concatenate([near, u_any])
    c["quat_ref"] = np.concatenate([zhat, ref_any])
    q = rng.standard_normal((n, 4))
    c["trafo_quat"] = q / np.linalg.norm(q, axis=1, keepdims=True)
    # getRotationMatrix normalises its own copy; Quaternion::rotate (and so
    # every trafo operation that rotates a vector) requires a unit quaternion
    c["rotmat_quat"] = c["trafo_quat"] * (1 + 1e-3 * rng.standard_normal((n, 1)))
    c["trafo_origin"] = rng.standard_normal((n, 3))
    c["trafo_r"] = 1e-3 * rng.standard_normal((n, 3))
    rq = rng.standard_normal((n, 4))
    c["right_quat"] = rq / np.linalg.norm(rq, axis=1, keepdims=True)
    c["right_origin"] = rng.standard_normal((n, 3))
    return c


def refpin():
    """refpin_kat.npz: the pinning cases and the answers of the reference's
    own BorisPusher, Quaternion and CoordinateSystemTrafo (compiled from
    source into oracle/_ref/librefpin.so)."""
    if not O.reference_pin_available():
        raise SystemExit("oracle/_ref/librefpin.so is missing: the reference tree is needed")
    c = pin_cases()
    ref = O.pin_cases_reference(c)
    np.savez_compressed(os.path.join(HERE, "refpin_kat.npz"), **{f"in_{k}": np.asarray(v) for k, v in c.items()},
                        **{f"ref_{k}": v for k, v in ref.items()})


if __name__ == "__main__":
    if sys.argv[1:] == ["refpin"]:
        O.build()
        refpin()
    else:
        main()
        refpin()
