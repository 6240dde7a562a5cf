"""The reference's file formats on the host side of the C ABI (no device):

* ASCII distribution of DISTRIBUTION TYPE=FROMFILE
  (src/Distribution/Distribution.cpp:1074-1159, converteVToBetaGamma :1047-1053);
* the SDDS statistics file of DataSink (src/Structure/DataSink.cpp:281-449,
  :585-1032), checked against the column table read from the reference's
  writer (tests/golden/sdds_stat_columns.json, made by make_golden.py).
"""
import json
import math
import os
import re

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def io():
    from src_b200 import scgpu
    scgpu.lib()
    return scgpu


def test_fromfile_round_trip_is_exact(io, tmp_path):
    rng = np.random.default_rng(3)
    R = rng.standard_normal((1001, 3)) * 1e-3
    P = rng.standard_normal((1001, 3))
    R[5] = (0.0, -0.0, 5e-324)
    path = tmp_path / "dist.txt"
    io.write_fromfile(path, R, P)
    R2, P2 = io.read_fromfile(path)
    np.testing.assert_array_equal(R2, R)
    np.testing.assert_array_equal(P2, P)
    first = path.read_text().splitlines()[:2]
    assert first[0] == "1001"
    vals = [float(v) for v in first[1].split()]
    assert vals == [R[0, 0], P[0, 0], R[0, 1], P[0, 1], R[0, 2], P[0, 2]]  # x px y py z pz


def test_fromfile_comments_and_layout(io, tmp_path):
    path = tmp_path / "dist.txt"
    path.write_text("# a distribution\n\n   # indented comment\n3   # particles\n"
                    "1 2 3 4 5 6\n7 8\n9 10 11 12\n 13 14 15 16 17 18 19\n")
    R, P = io.read_fromfile(path)
    np.testing.assert_array_equal(R, [[1, 3, 5], [7, 9, 11], [13, 15, 17]])
    np.testing.assert_array_equal(P, [[2, 4, 6], [8, 10, 12], [14, 16, 18]])


@pytest.mark.parametrize("text", ["0\n", "-4\n1 2 3 4 5 6\n", "   \n3\n", "x\n", "", "2\n1 2 3 4 5 6\n1 2 3\n"])
def test_fromfile_errors(io, tmp_path, text):
    path = tmp_path / "bad.txt"
    path.write_text(text)
    with pytest.raises(io.ScgpuError):
        io.read_fromfile(path)


def test_fromfile_ev_momenta(io, tmp_path):
    m = 0.51099892e6
    ev = np.array([[1e3, -2.5e6, 1e-9], [0.0, 3.0e-12, -7e5]])
    R = np.zeros_like(ev)
    path = tmp_path / "ev.txt"
    io.write_fromfile(path, R, ev)
    _, P = io.read_fromfile(path, momenta_in_ev=True, mass_ev=m)

    def conv(v):  # Distribution.cpp:1047-1053
        value = math.copysign(math.sqrt(math.pow(abs(v) / m + 1.0, 2.0) - 1.0), v)
        if abs(value) < np.finfo(float).eps:
            value = math.copysign(math.sqrt(2 * abs(v) / m), v)
        return value

    np.testing.assert_array_equal(P, np.vectorize(conv)(ev))


def _parse_sdds(text):
    blocks = re.findall(r"&(column|parameter|data|description)\n(.*?)&end\n", text, re.S)
    cols, params, data = [], [], []
    for kind, body in blocks:
        fields = dict(re.findall(r'\s*(\w+)=("[^"]*"|[^,\n]*),?\n', body))
        if kind == "column":
            cols.append([fields["name"], fields["type"], fields["units"], fields["description"].strip('"')])
        elif kind == "parameter":
            params.append([fields["name"], fields["type"]])
        elif kind == "data":
            data = [line.strip() for line in body.splitlines() if line.strip()]
    return cols, params, data


def test_sdds_header_matches_reference_writer(io, tmp_path):
    gold = json.load(open(os.path.join(GOLD, "sdds_stat_columns.json")))
    path = tmp_path / "run.stat"
    io.StatWriter(path, input_name="run.in", processors=1, revision="rev")
    text = path.read_text()
    assert text.startswith("SDDS1\n&description\n")
    cols, params, data = _parse_sdds(text)
    assert cols == gold["columns"]
    assert params == gold["parameters"]
    assert data == gold["data"]
    assert io.stat_column_names() == [c[0] for c in gold["columns"]]
    tail = text.split("&data\n", 1)[1].split("&end\n", 1)[1].splitlines()
    assert tail == ["1", "rev", "opal-t"]


def test_sdds_rows_format(io, tmp_path):
    path = tmp_path / "run.stat"
    w = io.StatWriter(path)
    row = np.arange(io.STAT_COLUMNS, dtype=float) * -1.25e-3
    row[2] = 1000000
    row[41] = 0
    w.write(row)
    w2 = io.StatWriter(tmp_path / "multi.stat", with_particle0=False)
    w2.write(row)
    line = path.read_text().splitlines()[-1]
    cells = line.split("\t")
    assert cells[-1] == ""  # every value is followed by the padded tab
    cells = cells[:-1]
    assert len(cells) == io.STAT_COLUMNS
    assert all(c.endswith(" " * 9) for c in cells)
    vals = [c.strip() for c in cells]
    assert vals[2] == "1000000" and vals[41] == "0"
    assert vals[0] == "-0.000000000000000e+00" and vals[1] == "-1.250000000000000e-03"
    # precision 15 in scientific notation: 16 significant digits, as the reference prints
    assert vals == [f"{v:.15e}" if i not in (2, 41) else str(int(v)) for i, v in enumerate(row)]
    assert len((tmp_path / "multi.stat").read_text().splitlines()[-1].split("\t")) == io.STAT_COLUMNS - 6 + 1
