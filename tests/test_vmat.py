"""The .vmat reader (ggi_tlm_b200/vmat.py) on the reference's own material
files (kept in tests/golden/vmat_text.npz by tests/golden/make_golden.py):
debye_2 must give the material the MATERIAL_STABILITY_TEST known-answer
case uses, whose probe series are pinned against the reference's golden
output; the others must give the coefficients their lines state."""
import os

import numpy as np
import pytest

from ggi_tlm_b200 import cases
from ggi_tlm_b200.problem import MAT_DISPERSIVE, material_coefficients
from ggi_tlm_b200.vmat import parse_vmat

HERE = os.path.dirname(os.path.abspath(__file__))


def files():
    d = np.load(os.path.join(HERE, "golden", "vmat_text.npz"))
    return {k: [str(x) for x in d[k]] for k in d.files}


def test_debye_2_is_the_stability_case_material():
    m, label, (fmin, fmax) = parse_vmat(files()["debye_2"])
    want = cases.debye_2()
    assert m.type == MAT_DISPERSIVE and label == "# debye dielectric model" and (fmin, fmax) == (0.0, 1e8)
    assert (m.eps.wnorm, list(m.eps.a), list(m.eps.b)) == (want.eps.wnorm, list(want.eps.a), list(want.eps.b))
    assert (m.mu.wnorm, list(m.mu.a), list(m.mu.b)) == (want.mu.wnorm, list(want.mu.a), list(want.mu.b))
    assert (m.sigma_e, m.sigma_m) == (want.sigma_e, want.sigma_m)
    # the same filter coefficients reach the tables
    a, b = material_coefficients(m, 1e-3, 1.6e-12), material_coefficients(want, 1e-3, 1.6e-12)
    assert a.keys() == b.keys() and all(np.array_equal(a[k], b[k]) for k in a)


def test_other_files():
    f = files()
    m1 = parse_vmat(f["debye_1"])[0]
    assert (m1.eps.wnorm, list(m1.eps.a), list(m1.eps.b), m1.sigma_e) == (1e8, [4.0, 0.75], [1.0, 0.5], 1.0)
    assert (list(m1.mu.a), list(m1.mu.b), m1.sigma_m) == ([3.0, 0.85], [1.0, 0.45], 10000.0)
    # order 0 with two numbers on the line: a list-directed read takes one and drops the rest
    m3 = parse_vmat(f["FR4_at_7GHz"])[0]
    assert (m3.eps.wnorm, list(m3.eps.a), list(m3.eps.b), m3.sigma_e) == (1.0, [4.45056], [1.0], 0.036549)


def test_truncated_file_is_an_error():
    with pytest.raises(ValueError):
        parse_vmat(files()["debye_1"][:9])
