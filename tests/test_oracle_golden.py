"""The CPU oracle against the reference's own golden time series.

The fixtures in tests/golden/ are the reference's TEST_DATA *.tout_ref files
(extracted by tests/golden/make_golden.py), printed with 8 significant digits
(format E16.7), so agreement is expected at ~1e-7 relative L2.
"""
import os

import numpy as np
import pytest

from ggi_tlm_b200 import cases
from ggi_tlm_b200.problem import build_tables, probe_series

import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL = 5e-7  # E16.7 print precision accumulated over the series


def golden(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    return d["time"], d["value"]


@pytest.mark.parametrize("name", sorted(cases.KAT_CASES))
def test_oracle_matches_reference_golden(name):
    spec = cases.KAT_CASES[name]()
    t = build_tables(spec)
    o = O.Oracle(t)
    ps = probe_series(t, o.run(t["n_timesteps"]))
    tr, vr = golden(name)
    v = np.where(np.abs(ps[0]) < 1e-30, 0.0, ps[0])  # output_points.F90:596-597
    assert len(v) == len(vr) == t["n_timesteps"]
    # output time stamps: time=(timestep-1)*dt
    np.testing.assert_allclose((np.arange(len(v))) * t["dt"], tr, rtol=1e-6, atol=1e-18)
    rel = np.linalg.norm(v - vr) / np.linalg.norm(vr)
    assert rel < TOL, rel


def test_material_changes_the_known_answer():
    """Without the Debye slab the TEM_MATERIAL series is far from golden, so
    the known answer pins the dispersive Z-filter path."""
    spec = cases.kat_tem_material()
    spec.materials, spec.material_regions = [], []
    t = build_tables(spec)
    ps = probe_series(t, O.Oracle(t).run(t["n_timesteps"]))
    _, vr = golden("tem_material_Ey")
    assert np.linalg.norm(ps[0] - vr) / np.linalg.norm(vr) > 0.05


def test_oracle_step_split_is_identical():
    """Running 2 x n steps equals one run of 2n steps (state carried exactly)."""
    spec = cases.pml_spheres(n=20, pml=4, n_spheres=2, steps=60, n_probes=3, n_freq=3, dft_size=6, rmin=2, rmax=3)
    t = build_tables(spec)
    a = O.Oracle(t)
    ca = np.concatenate([a.run(30), a.run(30)])
    b = O.Oracle(t)
    cb = b.run(60)
    assert np.array_equal(ca, cb)
    assert np.array_equal(a.dft(), b.dft())


def test_point_mapping_uses_reciprocal_multiply():
    """The MATERIAL_TEST2 source sits 4.2 mm from xmin, exactly on a cell
    boundary of 0.1 mm cells: int(4.2e-3/1e-4) is 41 but int(4.2e-3*(1/1e-4))
    is 42, and only the second one (cell 43) reproduces the golden series."""
    xmin, dl = -3.0e-3, cases.cubic_mesh_dl(-3.0e-3, 3.0e-3, 60)
    assert int((1.2e-3 - xmin) / dl) + 1 == 42
    assert cases.point_to_cell(1.2e-3, xmin, dl) == 43
    spec = cases.kat_material_test2()
    assert spec.point_excitations[0].cell == (43, 31, 31)
    assert spec.outputs[0].cell == (19, 31, 31)


def test_mesh_dl_uses_reciprocal_of_three():
    """On the HUYGENS_SURFACE mesh (4 m, 40 cells) (dlx+dly+dlz)/3 is one ulp
    above 0.1 and would put the output point (0,0,0) in cell 20; the
    reference's (dlx+dly+dlz)*(1/3) gives 0.1 and cell 21, which the golden
    series confirms."""
    dlx = 4.0 / 40
    assert (dlx + dlx + dlx) / 3.0 != 0.1
    assert cases.cubic_mesh_dl(-2.0, 2.0, 40) == 0.1
    assert cases.kat_huygens_box().outputs[0].cell == (21, 21, 21)


def _run_all(t, threads):
    o = O.Oracle(t, threads=threads)
    co = o.run(t["n_timesteps"])
    res = (co, o.links(), o.dft(), o.far_field(), o.face_probes())
    o.close()
    return res


@pytest.mark.parametrize("threads", [2, 3, 7])
def test_threaded_oracle_is_bit_identical(threads):
    """The oracle's plane-parallel scatter and connect (the CPU baseline's
    multi-core run) give the sequential results bit for bit: output cells,
    excitation cells, special faces with sources and outputs, PML, materials
    and far-field faces spread over planes that different threads take."""
    sys_path = os.path.join(os.path.dirname(__file__))
    import sys

    sys.path.insert(0, sys_path)
    import test_inp as T

    tabs = [build_tables(cases.pml_spheres(n=20, pml=4, n_spheres=3, steps=40, n_probes=4, n_freq=2, dft_size=6,
                                           rmin=2.0, rmax=3.0)),
            build_tables(cases.debye_slabs(nx=18, ny=16, nz=22, pml=4, n_slabs=2, thickness=2, steps=40)),
            build_tables(T.small(base=T.ALL_OUTPUTS).spec)]
    for t in tabs:
        a, b = _run_all(t, 1), _run_all(t, threads)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
