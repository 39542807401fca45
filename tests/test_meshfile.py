"""The mesh-file reader (ggi_tlm_b200/meshfile.py) on the reference's own
HELIX_ANTENNA/helix.mesh, as its mesher wrote it (kept as text in
tests/golden/mesh_text.npz by tests/golden/make_golden.py), and the .inp
reader taking its geometry from a mesh file: the volume as the mesher's cell
list (a rotated cylinder the package's own voxeliser refuses), the PEC
helices as face lists, the points on the mesh file's cells; the cables of
the same input stay refused."""
import os
import sys

import numpy as np
import pytest

from ggi_tlm_b200 import inp, meshfile
from ggi_tlm_b200.problem import CellList, UnsupportedFeature, build_tables

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import test_inp as T  # noqa: E402


def helix_mesh_lines():
    return [str(x) for x in np.load(os.path.join(HERE, "golden", "mesh_text.npz"))["helix"]]


def helix_inp_lines():
    return T.inputs()["helix"]


def test_helix_mesh_lists():
    m = meshfile.read_mesh(helix_mesh_lines())
    assert (m.dl, m.n) == (0.5, (42, 42, 42))
    assert m.extent == ((-10.5, 10.5),) * 3
    assert [v.shape for v in m.volumes] == [(1280, 4)]
    assert np.all(m.volumes[0][:, 3] == meshfile.CENTRE)
    assert m.volumes[0][0].tolist() == [20, 22, 17, 7]
    assert [s.faces.shape[0] for s in m.surfaces] == [6936, 1764, 4, 4, 43, 43]
    assert m.surfaces[1].cell_range == ((1, 42), (22, 22), (1, 42))
    assert [ln.shape for ln in m.lines] == [(10, 8), (10, 8)]
    assert len(m.points) == 4 and m.points[3].cell == (22, 24, 24) and m.points[0].face == (22, 22, 17, 1)
    assert not m.has_pml_section and m.pml_volumes == []


def test_the_cylinder_cells_lie_on_the_rotated_cylinder():
    """The volume is a cylinder of radius 2.5 m and height 8 m with its axis
    along y (Euler angles 90, 0, 90), centred at y = 4: every listed cell
    centre lies inside it, and nearly all cells whose centre lies well
    inside are listed."""
    m = meshfile.read_mesh(helix_mesh_lines())
    c = m.volumes[0][:, :3]
    x, y, z = (-10.5 + (c[:, a] - 0.5) * 0.5 for a in range(3))
    assert np.all(x ** 2 + z ** 2 <= 2.5 ** 2 + 1e-9) and np.all((y > 0.0) & (y < 8.0))
    g = np.stack(np.meshgrid(*(np.arange(1, 43),) * 3, indexing="ij"), -1).reshape(-1, 3)
    gx, gy, gz = (-10.5 + (g[:, a] - 0.5) * 0.5 for a in range(3))
    inside = (gx ** 2 + gz ** 2 < 2.2 ** 2) & (gy > 0.3) & (gy < 7.7)
    listed = {tuple(r) for r in c.tolist()}
    assert all(tuple(r) in listed for r in g[inside].tolist())


def test_records_ignore_labels_and_need_integers():
    lines = ["  0.1  dl", " 2 2 2  nx ny nz", " 0 0.2  x", " 0 0.2  y", " 0 0.2 z", " 1 n_volumes",
             " 2 number_of_cells", " 1 1 1 7", " 2 2 2 7", " 0 n_surfaces", " 0 n_lines", " 0 n_points"]
    m = meshfile.read_mesh(lines)
    assert m.volumes[0].tolist() == [[1, 1, 1, 7], [2, 2, 2, 7]]
    with pytest.raises(ValueError, match="integers"):
        meshfile.read_mesh(lines[:7] + [" 1.5 1 1 7"] + lines[8:])
    with pytest.raises(ValueError, match="ends early"):
        meshfile.read_mesh(lines[:-1])


def test_pml_section_and_shell_check():
    lines = ["  1.0  dl", " 4 4 4", " 0 4", " 0 4", " 0 4", " 0", " 0", " 0", " 0", " 1 n_pml_volumes"]
    shell = [(i, j, k) for k in range(1, 5) for j in range(1, 5) for i in range(1, 5)
             if min(i, j, k) == 1 or max(i, j, k) == 4]
    tail = [" pml_volume_to_face", " 1 2 3 4 5 6", " pml thicknesses", " 1.0 1.0", " 1.0 1.0", " 1.0 1.0",
            " pml reflection", " 1e-4 1e-4", " 1e-4 1e-4", " 1e-4 1e-4", " pml order", " 2"]
    m = meshfile.read_mesh(lines + [f" {len(shell)}"] + [f" {i} {j} {k} 7" for i, j, k in shell] + tail)
    assert m.has_pml_section and m.pml_order == 2 and m.pml_thickness == (1.0,) * 6
    assert meshfile.pml_cells_from_mesh(m) == (1,) * 6
    m2 = meshfile.read_mesh(lines + [f" {len(shell) - 1}"] + [f" {i} {j} {k} 7" for i, j, k in shell[1:]] + tail)
    with pytest.raises(UnsupportedFeature, match="box shell"):
        meshfile.pml_cells_from_mesh(m2)


def test_connect_faces():
    m = meshfile.MeshFile(dl=1.0, n=(4, 4, 4), extent=((0, 4),) * 3)
    f = np.array([[2, 2, 2, 1], [2, 2, 2, 4], [2, 3, 2, 5], [3, 3, 3, 3]], dtype=np.int32)
    assert meshfile.connect_faces(m, f, "s") == [((2, 2, 2), 1), ((3, 2, 2), 1), ((2, 4, 2), 2), ((3, 3, 3), 3)]
    with pytest.raises(ValueError, match="face code 7"):
        meshfile.connect_faces(m, np.array([[1, 1, 1, 7]]), "s")


def test_helix_input_with_its_mesh_refuses_the_cables():
    m = meshfile.read_mesh(helix_mesh_lines())
    with pytest.raises(UnsupportedFeature, match="cable"):
        inp.read_inp(helix_inp_lines(), T.materials, mesh_file=m)


def without_cables(lines):
    drop = {"line_list", "cable_geometry_list", "cable_list", "cable_output_list", "cable_junction_list"}
    out, skip = [], False
    for ln in lines:
        key = ln.strip().split()[0].lower() if ln.strip() else ""
        if key and not ln[:1].isspace() and key[0].isalpha() and key in inp.PACKETS:
            skip = key in drop
        if not skip:
            out.append(ln)
    return out


def test_helix_geometry_from_its_mesh_file():
    """Without its cables, the helix input reads with its mesh file: the
    dispersive volume is the mesher's 1280 cells of the rotated cylinder,
    the PEC surface material covers the two zplanes and the two helices
    face by face, and the output point sits on the mesh file's cell."""
    m = meshfile.read_mesh(helix_mesh_lines())
    lines = without_cables(helix_inp_lines())
    with pytest.raises(UnsupportedFeature, match="cylinder"):  # the package's own voxeliser refuses it
        inp.read_inp(lines, T.materials)
    p = inp.read_inp_lenient(lines, T.materials, mesh_file=m)
    s = p.spec
    (num, region), = s.material_regions
    assert num == 1 and isinstance(region, CellList) and region.cells.shape == (1280, 3)
    assert np.array_equal(region.cells, m.volumes[0][:, :3])
    assert s.outputs[0].cell == (22, 24, 24)
    assert [sh.kind for sh in s.surface_sheets] == ["PEC"] * 4
    assert [len(sh.faces) for sh in s.surface_sheets] == [4, 4, 43, 43]
    t = build_tables(s)
    assert int((np.asarray(t["sp_material"]) > 0).sum()) == 1280
    code = np.asarray(t["cell_code"]).reshape(42, 42, 42)
    mats = np.asarray(t["sp_material"])
    c = m.volumes[0]
    assert np.all(mats[code[c[:, 2] - 1, c[:, 1] - 1, c[:, 0] - 1] - 1] == 1)
    # the sheets' faces are the special faces with a PEC material; the helix surfaces share some faces
    keys = {k for sh in s.surface_sheets for k in sh.face_keys()}
    assert int(np.count_nonzero(np.asarray(t["face_mat"]) == 1)) == len(keys)


def test_mesh_file_must_match_the_problem():
    m = meshfile.read_mesh(helix_mesh_lines())
    m.n = (40, 42, 42)
    with pytest.raises(ValueError, match="do not match"):
        inp.read_inp(without_cables(helix_inp_lines()), T.materials, mesh_file=m)


@pytest.mark.gpu
def test_gpu_helix_from_its_mesh_matches_the_oracle(gpu_lib):
    """The helix problem read with its mesh file (cables left out, a soft Ez
    source at the dipole's centre instead): the mesher's dispersive
    cylinder, the PEC helices on their face lists, the far-field box, the
    output surface and the two frequency output surfaces (side -1) on the
    mesh file's faces; 300 FP64 steps on the GPU against the oracle on the
    same tables."""
    from ggi_tlm_b200 import capi

    sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
    import oracle

    from ggi_tlm_b200.problem import PointExcitation

    m = meshfile.read_mesh(helix_mesh_lines())
    spec = inp.read_inp_lenient(without_cables(helix_inp_lines()), T.materials, mesh_file=m).spec
    # the cables carried the problem's only source: drive the dipole's centre cell instead
    spec.point_excitations.append(PointExcitation(m.points[1].cell, "Ez", 1))
    t = build_tables(spec)
    n = 300
    o = oracle.Oracle(t, threads=4)
    want = o.run(n)
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.run(n)
        got, links, dft, ff = g.cell_output(1, n), g.links(), g.dft(), g.far_field()
    assert np.linalg.norm(got - want) <= 1e-10 * np.linalg.norm(want)
    assert np.linalg.norm(links - o.links()) <= 1e-10 * np.linalg.norm(o.links())
    assert np.linalg.norm(dft - o.dft()) <= 1e-10 * np.linalg.norm(o.dft())
    assert np.linalg.norm(ff - o.far_field()) <= 1e-10 * np.linalg.norm(o.far_field())
    o.close()
