"""The .tout writer (ggi_tlm_b200/tout.py): the reference's own .tout_ref
files (header and every data line, kept in tests/golden/tout_text.npz by
tests/golden/make_golden.py) are reproduced byte for byte from their
numbers, and a file written from the oracle's series reads back to them in
the reference's line order and numbering."""
import os
import sys

import numpy as np

from ggi_tlm_b200 import cases, tout
from ggi_tlm_b200.problem import OutputPoint, build_tables, probe_series

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import oracle  # noqa: E402


def test_reference_lines_byte_for_byte():
    d = np.load(os.path.join(HERE, "golden", "tout_text.npz"))
    n_lines = 0
    for name in d.files:
        lines = [str(x) for x in d[name]]
        hdr, data = lines[:3], lines[3:]
        n_pts, n_steps = int(hdr[1].split(":")[1]), int(hdr[2].split(":")[1])
        assert tout.header(n_pts, n_steps) == hdr, name
        for line in data:
            t, p, v = line.split()
            assert tout.data_line(float(t), int(p), float(v)) == line, (name, line)
        n_lines += len(data)
    assert n_lines > 7000


def test_fortran_e_edges():
    assert tout.fortran_e(0.0) == "   0.0000000E+00"
    assert tout.fortran_e(-1.0) == "  -0.1000000E+01"
    assert tout.fortran_e(9.99999995e-3) == "   0.1000000E-01"  # rounding carries into the exponent
    assert tout.fortran_e(1.5e-120) == "   0.1500000-119"     # three-digit exponents drop the E
    assert tout.data_line(1e-9, 3, 5e-31) == "   0.1000000E-08    3   0.0000000E+00"  # below 1e-30 -> 0


def test_field_file_from_oracle_series(tmp_path):
    spec = cases.pml_point_source(16, pml=3, steps=30, n_probes=0)
    spec.outputs = [OutputPoint((8, 8, 10), "Ex"), OutputPoint((5, 6, 7), "Ey", face="xmin"),
                    OutputPoint((9, 9, 9), "Hz")]
    t = build_tables(spec)
    o = oracle.Oracle(t)
    centre = probe_series(t, o.run(t["n_timesteps"]))
    face = o.face_probes()
    rows = tout.field_rows(t, centre, face)
    path = os.path.join(tmp_path, "x.field.tout")
    tout.write_tout(path, rows, n_points=3, n_timesteps=t["n_timesteps"])
    back = tout.read_tout(path)
    assert back.shape == (3 * 30, 3)
    assert list(back[:3, 1]) == [1, 3, 2]  # centre points, then the face point half a step later
    assert back[0, 0] == 0.0 and abs(back[2, 0] - t["dt"] / 2.0) <= 1e-7 * t["dt"]  # 7 significant digits
    want = np.array([v for _, _, v in rows])
    want[np.abs(want) < 1e-30] = 0.0
    assert np.allclose(back[:, 2], want, rtol=5.01e-7, atol=0)  # 0.ddddddd: half a unit of the 7th digit
    with open(path) as f:
        assert f.readline().rstrip("\n") == tout.HEADER


def test_non_finite_values():
    from ggi_tlm_b200.tout import fortran_e

    assert fortran_e(float("-inf")) == "       -Infinity"
    assert fortran_e(float("inf")) == "        Infinity"
    assert fortran_e(float("nan")) == "             NaN"
