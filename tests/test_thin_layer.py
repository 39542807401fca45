"""Dispersive thin-layer surface materials (surface_material_type_DISPERSIVE
and ANISOTROPIC_DISPERSIVE): the two-port impedance update of
MATERIALS/TLM_surface_materials.F90:535-697 in the connect of the faces a
layer covers (connect_normal_to_x.F90:268-282 and the y, z analogues).

The reference's eight thin-layer cases are read from their own input files
with their .smat files and run on the oracle against their golden series:
TEM_THIN_LAYER_TEST (an isotropic dispersive sheet across a TEM column),
the six anisotropic sheets across x-, y- and z-directed columns with the
two transverse polarisations each, and THIN_LAYER_STABILITY_TEST (a sheet
inside a cavity, 5996 steps).  GPU: the library against the oracle."""
import os
import sys

import numpy as np
import pytest

from ggi_tlm_b200 import capi, inp
from ggi_tlm_b200.problem import build_tables, probe_series
from ggi_tlm_b200.smat import parse_smat

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import test_inp as T  # noqa: E402
import oracle  # noqa: E402

CASES = ["tem_thin_layer", "tem_x_aniso_y", "tem_x_aniso_z", "tem_y_aniso_x", "tem_y_aniso_z", "tem_z_aniso_x",
         "tem_z_aniso_y", "thin_layer_stability"]
TOL = 5e-7  # the golden series' E16.7 print precision


def thin_layer(name, anisotropic):
    d = np.load(os.path.join(HERE, "golden", "smat_text.npz"))
    return parse_smat([str(x) for x in d[name.split("/")[-1]]], anisotropic)[0]


def tables(case):
    return build_tables(inp.read_inp(T.inputs()[case], T.materials, thin_layer=thin_layer).spec)


def test_smat_reader():
    d = np.load(os.path.join(HERE, "golden", "smat_text.npz"))
    iso, label, frange = parse_smat([str(x) for x in d["Dispersive_sheet"]])
    assert frange == (0.0, 1e8) and label.startswith("# dispersive")
    f = iso.z[0][0]
    assert (f.wnorm, f.a, f.b) == (1e8, [377.0, 100.0], [1.0, 0.75])
    assert all(iso.z[p][k] == f for p in range(3) for k in range(4))
    an = parse_smat([str(x) for x in d["Anisotropic_sheet"]], anisotropic=True)[0]
    assert [an.z[p][0].a[0] for p in range(3)] == [188.5, 377.0, 754.0]


def test_tables_mark_the_sheet_faces():
    t = tables("tem_thin_layer")
    mat = np.asarray(t["face_mat"])
    assert int(t["n_smat"]) == 1 and int(np.count_nonzero(mat == 3)) == 1
    assert int(np.asarray(t["face_smat"])[mat == 3][0]) != 0
    assert t["smat_order"].shape == (1, 3, 4) and int(t["smat_order"].max()) == 1


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_the_reference_thin_layer_cases(case):
    t = tables(case)
    g = np.load(os.path.join(HERE, "golden", case + ".npz"))
    series = probe_series(t, oracle.Oracle(t).run(t["n_timesteps"]))
    for pt in np.unique(g["point"]):
        want = g["value"][g["point"] == pt]
        v = np.where(np.abs(series[pt - 1]) < 1e-30, 0.0, series[pt - 1])
        assert len(v) == len(want)
        assert np.linalg.norm(v - want) / np.linalg.norm(want) < TOL


def test_the_layer_changes_the_field():
    """Without the sheet the TEM column's golden series is far off: the
    golden vector really pins the thin-layer update."""
    p = inp.read_inp(T.inputs()["tem_thin_layer"], T.materials, thin_layer=thin_layer)
    p.spec.surface_sheets = []
    t = build_tables(p.spec)
    g = np.load(os.path.join(HERE, "golden", "tem_thin_layer.npz"))
    v = probe_series(t, oracle.Oracle(t).run(t["n_timesteps"]))[0]
    assert np.linalg.norm(v - g["value"]) / np.linalg.norm(g["value"]) > 0.05


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["tem_thin_layer", "tem_y_aniso_z", "tem_z_aniso_x", "thin_layer_stability"])
def test_gpu_thin_layer_matches_the_oracle(gpu_lib, case):
    """The links are compared a quarter of the way in, while the pulse is in
    the mesh, and at the end against that scale: by the last step the pulse
    has left the TEM column and the links that remain are ~1e-15 of it, so
    rounding noise is all a comparison relative to them would see."""
    t = tables(case)
    o = oracle.Oracle(t)
    n1 = int(t["n_timesteps"]) // 4
    want = o.run(n1)
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.run(n1)
        mid = o.links()
        scale = np.linalg.norm(mid)
        assert scale > 0
        assert np.linalg.norm(g.links() - mid) <= 1e-10 * scale
        want = np.concatenate([want, o.run(int(t["n_timesteps"]) - n1)])
        g.run(int(t["n_timesteps"]) - n1)
        got, links = g.cell_output(), g.links()
    assert got.shape == want.shape
    assert np.linalg.norm(got - want) <= 1e-10 * np.linalg.norm(want)
    assert np.linalg.norm(links - o.links()) <= 1e-10 * scale
    o.close()
