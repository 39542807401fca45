"""The .inp reader (ggi_tlm_b200/inp.py) on the reference's own problem
input files (kept as text in tests/golden/inp_text.npz by
tests/golden/make_golden.py) and on small inputs written here.

The five known-answer inputs must give tables equal, array for array, to
the hand-built known-answer specs, whose probe series the oracle pins
against the reference's golden output; the HUYGENS_SURFACE input, read
whole (30 output points, 3 output surfaces, 3 output volumes), must
reproduce all six golden centre series through the oracle.  The small
inputs check the reader's rules one at a time: Fortran reals, packet
keywords, plane orientation, output timing, refusals.  GPU: the whole
HUYGENS_SURFACE input against the oracle."""
import os
import sys

import numpy as np
import pytest

from ggi_tlm_b200 import capi, cases, inp
from ggi_tlm_b200.problem import (Z0, HuygensOuter, HuygensPlane, UnsupportedFeature, build_tables,
                                  material_coefficients, probe_series)
from ggi_tlm_b200.tout import field_rows, output_flag
from ggi_tlm_b200.vmat import parse_vmat

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import oracle  # noqa: E402

KAT = {"tem_pml": "tem_pml_Ey", "tem_material": "tem_material_Ey", "material_stability": "material_stability_Ey",
       "material_test2": "material_test2_Ex", "huygens_box": "huygens_box_Ex"}
TOL = 5e-7  # the golden series' E16.7 print precision


def inputs():
    d = np.load(os.path.join(HERE, "golden", "inp_text.npz"))
    return {k: [str(x) for x in d[k]] for k in d.files}


def materials(name):
    """The material resolver: MATERIAL_DIRECTORY/<name> -> the fixture's .vmat text."""
    d = np.load(os.path.join(HERE, "golden", "vmat_text.npz"))
    return parse_vmat([str(x) for x in d[name.split("/")[-1]]])[0]


def read(name):
    return inp.read_inp(inputs()[name], materials)


def same_tables(a, b):
    keys = set(a) | set(b)
    return [k for k in keys if k not in a or k not in b or
            np.asarray(a[k]).shape != np.asarray(b[k]).shape or not np.array_equal(np.asarray(a[k]), np.asarray(b[k]))]


@pytest.mark.parametrize("name", sorted(KAT))
def test_known_answer_inputs_give_the_known_answer_tables(name):
    p = read(name)
    spec = p.spec
    if name == "huygens_box":  # the known-answer spec keeps output point 1 only
        assert len(spec.outputs) == 30 and len(spec.output_surfaces) == 3 and len(spec.output_volumes) == 3
        spec.outputs, spec.output_surfaces, spec.output_volumes = spec.outputs[:1], [], []
    assert p.skipped == []
    assert same_tables(build_tables(spec), build_tables(cases.KAT_CASES[KAT[name]]())) == []


def test_lorentz_material_file_is_the_known_answer_material():
    a = material_coefficients(materials("MATERIAL_DIRECTORY/mur_lorentz"), 1e-4, 1e-4 / (2 * 299792458.0))
    want = cases.kat_material_test2().materials[0]
    b = material_coefficients(want, 1e-4, 1e-4 / (2 * 299792458.0))
    assert a.keys() == b.keys() and all(np.array_equal(a[k], b[k]) for k in a)


def test_huygens_input_reproduces_all_golden_centre_series():
    """Output points 1, 6, 11, 16, 21, 26 of huygens_test.inp are Ex..Hz at
    the centre; the face points and the output surfaces and volumes ride
    along in the same run."""
    p = read("huygens_box")
    t = build_tables(p.spec)
    assert list(t["out_point_no"]) == [1, 6, 11, 16, 21, 26]
    assert int(t["n_face_probes"]) == 24
    series = probe_series(t, oracle.Oracle(t).run(t["n_timesteps"]))
    for k, comp in enumerate(("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")):
        g = np.load(os.path.join(HERE, "golden", f"huygens_box_{comp}.npz"))
        v = np.where(np.abs(series[k]) < 1e-30, 0.0, series[k])
        assert np.linalg.norm(v - g["value"]) / np.linalg.norm(g["value"]) < TOL, comp


def test_huygens_input_output_surfaces_and_volumes():
    """The xplane/yplane/zplane output surfaces with side -1 over the whole
    mesh, Emagnitude on steps 1, 5, ..., 117 (first step 0 raised to 1), and
    the 2 x 2 x 0.1 m output volume: one layer of 20 x 20 cells at z = 0.05."""
    p = read("huygens_box")
    s1, s2, s3 = p.spec.output_surfaces
    # xplane and zplane corners ascending: normal +axis, so side -1 samples the faces of HuygensPlane side 1;
    # yplane corners ascending: normal -y, so side -1 samples side -1
    assert (s1.plane, s1.side) == ((1, 20, (1, 40), (1, 40)), 1)
    assert (s2.plane, s2.side) == ((2, 20, (1, 40), (1, 40)), -1)
    assert (s3.plane, s3.side) == ((3, 20, (1, 40), (1, 40)), 1)
    assert all((s.component, s.first_step, s.last_step, s.interval, s.both_sides) == ("Em", 1, 120, 4, False)
               for s in (s1, s2, s3))
    v = p.spec.output_volumes
    assert [o.component for o in v] == ["Hx", "Hy", "Hz"]
    b = v[0].region
    assert (b.i0, b.i1, b.j0, b.j1, b.k0, b.k1) == (11, 30, 11, 30, 21, 21)
    t = build_tables(p.spec)
    shapes = capi.output_surface_shapes(t)
    assert shapes == [(30, 1600)] * 3


# ---------------------------------------------------------------------------
# the reader's rules on small inputs
# ---------------------------------------------------------------------------
BASE = """# a small test problem
Mesh_outer_boundary_dimension
0.0 1.0  0.0 1.0  0.0 1.0
Mesh_cell_dimension
0.1
Point_list
1
1
0.55 0.55 0.55
0 0 0
0 0 0
Excitation_function_list
1
1
gaussian
1.0 1e-9 3e-9
Simulation_time
1e-8
"""


def small(extra="", base=BASE):
    return inp.read_inp((base + extra).splitlines(), materials)


def test_required_packets():
    with pytest.raises(ValueError, match="no simulation_time packet"):
        small(base=BASE.replace("Simulation_time\n1e-8\n", ""))
    with pytest.raises(ValueError, match="no mesh_outer_boundary_dimension packet"):
        inp.read_inp(["# the input of another program", "Filter_order", "2"], materials)


def test_every_keyword_has_one_treatment():
    groups = [inp.HANDLED, inp.NEUTRAL, inp.UNSUPPORTED, inp.NOT_READ]
    assert set().union(*groups) == inp.PACKETS
    assert sum(len(g) for g in groups) == len(inp.PACKETS)


def test_fortran_reals():
    assert inp.fortran_real("3.0-3") == 3.0e-3
    assert inp.fortran_real("1.5d+2") == 150.0
    assert inp.fortran_real("2E1") == 20.0
    assert inp.fortran_real(".5") == 0.5 and inp.fortran_real("5.") == 5.0 and inp.fortran_real("-7") == -7.0
    for bad in ("x", "1.0e", "--1", "1,0"):
        with pytest.raises(ValueError):
            inp.fortran_real(bad)
    # list-directed: values spill over lines, the rest of the last line is ignored, r*c repeats c
    r = inp.Records("t", ["1 2", "4,5 6 ! remark", "2*0.5 remark"])
    assert r.values(4) == [1.0, 2.0, 4.0, 5.0] and r.values(2) == [0.5, 0.5]
    with pytest.raises(ValueError, match="expected a number"):
        inp.Records("t", ["1 2 ! remark 3"]).values(3)


def test_packet_keywords():
    pk = inp.split_packets(["title line", "MESH_CELL_DIMENSION   ! remark", "0.1", "", "simulation_time",
                            "pml 3 cells", "1e-8"])
    assert pk == [("mesh_cell_dimension", ["0.1"]), ("simulation_time", ["pml 3 cells", "1e-8"])]


def test_small_problem_mesh_time_and_points():
    p = small("""Excitation_point_list
1
1
1
1
Jz
xmax
hard
Output_point_list
2
1
1
Ey
centre
output_time_information
2e-9
5e-9
0.5e-9
2
1
Hx
zmin
output_timestep_information
0
7
3
""")
    s = p.spec
    assert (s.nx, s.ny, s.nz, s.dl) == (10, 10, 10, 0.1)
    dt = 0.1 / (2 * 299792458.0)
    assert s.n_timesteps == round(1e-8 / dt)
    e = s.point_excitations[0]
    assert (e.cell, e.component, e.face, e.source_type) == ((6, 6, 6), "Jz", "xmax", 0)
    assert [(o.cell, o.component, o.face) for o in s.outputs] == [((6, 6, 6), "Ey", "centre"), ((6, 6, 6), "Hx", "zmin")]
    assert p.output_timing == [(round(2e-9 / dt), round(5e-9 / dt), round(0.5e-9 / dt)), (1, 7, 3)]
    assert [ts for ts in range(1, 12) if output_flag(ts, p.output_timing[1])] == [1, 4, 7]


def test_cell_count_mesh_and_pml():
    base = BASE.replace("Mesh_cell_dimension\n0.1\n", "Mesh_dimensions_in_cells\n20 20 20\n")
    p = small("""PML
0.2   ! the same thickness on every side
1e-3 1e-3 1e-3 1e-3 1e-3 1e-2
3
""", base)
    s = p.spec
    assert (s.nx, s.dl) == (20, 0.05)
    assert s.pml_cells == (4,) * 6 and s.pml_r == (1e-3,) * 5 + (1e-2,) and s.pml_order == 3
    # a cell size wins over a cell count
    both = BASE + "Mesh_dimensions_in_cells\n20 20 20\n"
    assert small("", both).spec.nx == 10


def test_plane_orientation_and_huygens_variants():
    surf = """Surface_list
3
1
zplane
0.0 0.0 0.5   1.0 1.0 0.5
0 0 0
0 0 0
2
zplane
1.0 0.0 0.5   0.0 1.0 0.5
0 0 0
0 0 0
3
rectangle
1.0 1.0
0 0 0
0.5 0.5 0.5
"""
    hs = "Huygens_surface\n{n}\n1\n{z}1\n0.0 0.0\n1.0 0.0\n"
    got = {}
    for n in (1, 2, 3):
        got[n] = small(surf + hs.format(n=n, z="")).spec.huygens
        assert isinstance(got[n], HuygensPlane) and (got[n].axis, got[n].index) == (3, 5)
    # ascending zplane corners: normal +z, the other side of the rectangle's -z; swapping x flips it back
    assert (got[1].side, got[2].side, got[3].side) == (-1, 1, 1)
    # a wave impedance other than Z0 scales H only
    t0 = build_tables(small(surf + hs.format(n=3, z="")).spec)
    t1 = build_tables(small(surf + hs.format(n=3, z="wave_impedance\n100.0\n")).spec)
    assert np.array_equal(t0["hs_Ei"], t1["hs_Ei"])
    assert np.allclose(t1["hs_Hi"], t0["hs_Hi"] * (Z0 / 100.0), rtol=1e-15, atol=0)
    assert isinstance(small(hs.format(n=0, z="")).spec.huygens, HuygensOuter)
    with pytest.raises(UnsupportedFeature):
        small(surf + "Huygens_surface\n3\n1\n1\nrandom\n1.0 0.0\n")
    with pytest.raises(ValueError):
        small(surf + "Huygens_surface\n3\n2\n1\n0.0 0.0\n1.0 0.0\n")


def test_output_surface_both_sides_and_volumes():
    geo = """Volume_list
1
1
rectangular_block
0.4 0.4 0.4
0 0 0
0.5 0.5 0.5
Surface_list
1
1
rectangular_block
0.4 0.4 0.4
0 0 0
0.5 0.5 0.5
"""
    p = small(geo + """Output_surface_list
2
1
1
0
Jmagnitude
2
1
1
Hy
output_timestep_information
2
10
2
Output_volume_list
1
1
1
Ez
""")
    a, b = p.spec.output_surfaces
    assert (a.component, a.side, a.both_sides, a.box) == ("Jm", -1, True, ((4, 7), (4, 7), (4, 7)))
    assert (b.component, b.side, b.first_step, b.last_step, b.interval) == ("Hy", 1, 2, 10, 2)
    v = p.spec.output_volumes[0]
    assert (v.component, v.kind, v.first_step, v.last_step, v.region.i0, v.region.i1) == ("Ez", "field", 1, None, 4, 7)
    with pytest.raises(ValueError):  # both sides is for J only
        small(geo + "Output_surface_list\n1\n1\n1\n0\nEx\n")


@pytest.mark.parametrize("extra, match", [
    ("Volume_list\n1\n1\nrectangular_block\n0.4 0.4 0.4\n0 0 45\n0.5 0.5 0.5\nVolume_material_list\n1\n1\nPEC\n1\n1\n",
     "rotated rectangular_block"),                                                             # rotated, used
    ("Volume_list\n1\n1\nrectangular_block\n0.4 0.4 0.4\n0 0 45\n0.5 0.5 0.5\n", None),    # rotated, unused
    ("Volume_list\n1\n1\nsphere\n0.2\n0 0 0\n0.5 0.5 0.5\nVolume_material_list\n1\n1\nPEC\n1\n1\n",
     "type 'sphere'"),                                                                      # not voxelised here
    ("Volume_list\n1\n1\nrectangular_block\n0.5 0.5 0.5\n0 0 0\n0.5 0.5 0.5\nVolume_material_list\n1\n1\nPEC\n1\n1\n",
     "centre lies on"),                                                                      # a face through centres
    ("Surface_list\n1\n1\nrectangle\n1.0 1.0\n0 0 0\n0.5 0.5 0.5\nSurface_material_list\n1\n1\nDIODE\n"
     "1e-14 0.025 1.0 1e-12 +x\n1\n1\n1\n", "surface material 'diode'"),
    ("Surface_list\n1\n1\nrectangle\n1.0 1.0\n0 0 0\n0.5 0.5 0.5\nSurface_material_list\n1\n1\nDISPERSIVE\n"
     "MATERIAL_DIRECTORY/sheet\n1\n1\n1\n", "no surface material file resolver"),
    ("Cable_list\n0\n", "cable_list packet"),
    ("Output_mode_list\n1\n1\n1\n1\nEx\nWR90.mode\n1\n2\n3\n6\n", "no file opener"),          # mode file
    ("Frequency_scale_flag\nT\n2.0\n", "frequency scale"),
    ("Bicubic_warp_flag\n.true.\n", "bicubic"),
    ("Excitation_function_list\n1\n1\nnoise\n1.0\n", "function 'noise'"),
    ("Output_point_list\n1\n2\n1\nEx\ncentre\n", "numbered in order"),                                  # numbering
    ("Output_point_list\n1\n1\n1\nJx\ncentre\n", "component 'jx'"),                                  # not a field
    ("Surface_list\n1\n1\nrectangle\n1.0 1.0\nsurface_roughness\n0.01 0.1\n0 0 0\n0.5 0.5 0.5\n"
     "Huygens_surface\n1\n1\n1\n0 0\n1 0\n", "roughness"),                               # random roughness
])
def test_refusals(extra, match):
    """Inputs the GPU path cannot run exactly raise UnsupportedFeature; a
    malformed input raises ValueError, as the reference stops with an error."""
    base = BASE.replace("Excitation_function_list\n1\n1\ngaussian\n1.0 1e-9 3e-9\n", "") \
        if "Excitation_function_list" in extra else BASE
    if match is None:  # refused only where it is used
        small(extra, base)
        return
    err = ValueError if match in ("numbered in order", "component 'jx'") else UnsupportedFeature
    with pytest.raises(err, match=match) as e:
        small(extra, base)
    assert (e.type is UnsupportedFeature) == (err is UnsupportedFeature)


def test_neutral_packets_are_listed_and_pec_materials():
    p = small("""New_mesh_generation
No_geometry_vtk_files
Far_field_surface_list
0
Volume_list
1
1
rectangular_block
0.4 0.4 0.4
0 0 0
0.5 0.5 0.5
Volume_material_list
1
1
PMC
1
1
Bicubic_warp_flag
F
""")
    assert p.skipped == ["new_mesh_generation", "no_geometry_vtk_files"]
    assert p.spec.far_field_surfaces == [] and p.post["far_field"] == []
    assert p.spec.materials[0].type == 2 and p.spec.material_regions[0][1].i0 == 4


def test_field_rows_follow_output_timing():
    p = small("""Output_point_list
2
1
1
Ex
centre
output_timestep_information
2
6
2
2
1
Ey
centre
""")
    p.spec.n_timesteps = 8
    t = build_tables(p.spec)
    centre = np.arange(16, dtype=float).reshape(2, 8) + 1.0
    rows = field_rows(t, centre, np.zeros((0, 8)), timing=p.output_timing)
    assert [(r[1], round(r[0] / t["dt"]) + 1) for r in rows if r[1] == 1] == [(1, 2), (1, 4), (1, 6)]
    assert sum(1 for r in rows if r[1] == 2) == 8


@pytest.mark.gpu
def test_gpu_huygens_input_matches_oracle(gpu_lib):
    p = read("huygens_box")
    t = build_tables(p.spec)
    o = oracle.Oracle(t)
    want = o.run(t["n_timesteps"])
    want_faces = o.face_probes()
    want_surf = oracle.output_surfaces(t)
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.run(t["n_timesteps"])
        got, faces, surf = g.cell_output(), g.face_output(), g.output_surfaces()
    for a, b in zip(probe_series(t, got), probe_series(t, want)):
        assert np.linalg.norm(a - b) <= 1e-10 * np.linalg.norm(b)
    assert np.linalg.norm(faces - want_faces) <= 1e-10 * np.linalg.norm(want_faces)
    for a, b in zip(surf, want_surf):
        assert a.shape == b.shape and np.linalg.norm(a - b) <= 1e-10 * np.linalg.norm(b)


ALL_OUTPUTS = BASE.replace("0.55 0.55 0.55", "0.15 0.15 0.15") + """Volume_list
1
1
rectangular_block
0.4 0.4 0.4
0 0 0
0.5 0.5 0.5
Surface_list
3
1
rectangular_block
0.6 0.6 0.6
0 0 0
0.5 0.5 0.5
2
zplane
0.2 0.2 0.3   0.8 0.8 0.3
0 0 0
0 0 0
3
rectangle
0.6 0.6
0 0 0
0.5 0.5 0.7
Volume_material_list
1
1
dispersive
MATERIAL_DIRECTORY/debye_2
1
1
Surface_material_list
2
1
free_space
1
1
1
2
PEC
1
2
-1
Excitation_point_list
1
1
1
1
Ez
centre
soft
Output_point_list
1
1
1
Ez
centre
Output_volume_average_list
1
1
1
Ex
output_timestep_information
2
20
3
Output_volume_peak_list
1
1
1
Hz
Frequency_output_volume_list_xyz
1
output_every 2
1
1
1e8
Ey
Frequency_output_surface_list
1
1
3
1
2e8
Jx
Far_field_surface_list
1
1
1
1
3e8
0 180 5
0 90 10
2D
z
RCS_surface
1
-1
1e8 5e8 1e8
90.0
0.0
Frequency_domain_power_surface_list
1
1
2
1
1e8 3e8 3
SAR_volume_list
1
1
1
1e8
1000.0
"""


def test_all_output_packets():
    p = small(base=ALL_OUTPUTS)
    s = p.spec
    blk = (4, 7, 4, 7, 4, 7)
    cells = lambda b: (b.i0, b.i1, b.j0, b.j1, b.k0, b.k1)  # noqa: E731
    assert [(v.kind, v.component, v.first_step, v.last_step, v.interval, cells(v.region)) for v in s.output_volumes] \
        == [("average", "Ex", 2, 20, 3, blk), ("peak", "Hz", 1, None, 1, blk)]
    fv = s.frequency_output_volumes[0]
    assert (list(fv.frequencies), fv.component, fv.every, cells(fv.region)) == ([1e8], "Ey", 2, blk)
    ds = s.dft_surfaces[0]
    assert (ds.axis, ds.index, ds.r0, ds.r1, list(ds.frequencies), ds.component) == (3, 7, (3, 8), (3, 8), [2e8], "Jx")
    ff = s.far_field_surfaces[0]
    assert (ff.frequencies, ff.box, ff.side) == ([3e8], ((3, 8), (3, 8), (3, 8)), 1)
    assert p.post["far_field"][0]["dim"] == 2 and p.post["far_field"][0]["phi"] == (0.0, 90.0, 10.0)
    rc = s.rcs_surface
    assert (rc.theta, rc.phi, rc.box, rc.side, p.post["rcs"]) == (90.0, 0.0, ((3, 8), (3, 8), (3, 8)), -1,
                                                                  (1e8, 5e8, 1e8))
    ps = s.power_surfaces[0]
    # ascending zplane corners: normal +z, so side 1 of the packet is side -1 of the spec
    assert (ps.frequencies, ps.plane, ps.side) == ([1e8, 2e8, 3e8], (3, 3, (3, 8), (3, 8)), -1)
    assert (list(s.sar_volumes[0].frequencies), cells(s.sar_volumes[0].region), p.post["sar_density"]) == \
        ([1e8], blk, [1000.0])
    kinds = [(sh.kind, sh.axis, sh.index) for sh in s.surface_sheets]
    assert kinds == [("free", 1, 2), ("free", 1, 8), ("free", 2, 2), ("free", 2, 8), ("free", 3, 2), ("free", 3, 8),
                     ("PEC", 3, 3)]
    t = build_tables(s)
    assert (t["n_ovol"], t["n_vdft"], t["n_dft"], t["n_sar"], t["n_ff"], t["n_ps"]) == (2, 1, 1, 1, 1, 3)
    assert int(np.count_nonzero(t["face_mat"])) == 6 * 36 + 36  # free-space box faces and the PEC sheet


@pytest.mark.gpu
def test_gpu_all_output_packets_match_oracle(gpu_lib):
    t = build_tables(small(base=ALL_OUTPUTS).spec)
    o = oracle.Oracle(t)
    want = o.run(t["n_timesteps"])
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.run(t["n_timesteps"])
        got, got_dft, got_ps, got_ov = g.cell_output(), g.dft(), g.power_surfaces(), g.output_volumes()

    def rel(a, b):
        assert a.shape == b.shape
        return np.linalg.norm(a - b) / np.linalg.norm(b)

    # only the output point keeps a time series; the volume outputs' cells
    # report through their own accumulators, checked below
    keep = np.asarray(t["out_keep"]) == 1
    assert got.shape == (t["n_timesteps"], int(keep.sum()), 6)
    assert rel(got, want[:, keep, :]) < 1e-10
    assert rel(got_dft, o.dft()) < 1e-10
    want_ps, ptr = oracle.power_surfaces(t), t["ps_face_ptr"]
    for k in range(t["n_ps"]):
        assert rel(got_ps[ptr[k]:ptr[k + 1]], want_ps[ptr[k]:ptr[k + 1]]) < 1e-10, k
    for a, b in zip(got_ov, oracle.output_volumes(t, want)):
        assert a.shape == b.shape and rel(a, b) < 1e-10


def data_file(name):
    d = np.load(os.path.join(HERE, "golden", "data_text.npz"))
    return [str(x) for x in d[name]]


def test_interpolate_function():
    from ggi_tlm_b200.problem import interpolate_function

    ts, vs = [0.0, 1.0, 3.0], [2.0, 4.0, 0.0]
    assert interpolate_function(-1.0, ts, vs) == 2.0 and interpolate_function(5.0, ts, vs) == 0.0
    assert interpolate_function(1.0, ts, vs) == 4.0  # a sample time: the first interval holding it
    assert interpolate_function(0.5, ts, vs) == 3.0 and interpolate_function(2.0, ts, vs) == 2.0


def test_excitation_function_from_a_file_reproduces_the_golden_field():
    """EXCITATION_FUNCTION_TEST: a Gaussian read from gaussian_from_file.dat
    (240 samples, amplitude 5, delay 1 ns) launched by a closed Huygens box;
    the centre Ex series against excitation_test.field.tout_ref."""
    p = inp.read_inp(inputs()["excitation_test"], materials, data_file)
    f = p.spec.functions[0]
    assert (f.type, f.parameters, len(f.samples[0])) == ("file", (5.0, 1e-9), 240)
    t = build_tables(p.spec)
    assert t["n_timesteps"] == 300
    # the tabulated values are the interpolated samples, scaled and delayed, at (ts-1)*dt
    from ggi_tlm_b200.problem import interpolate_function

    val = np.asarray(t["fn_value"]).reshape(-1)
    for ts in (1, 40, 100, 300):
        assert val[ts - 1] == 5.0 * interpolate_function((ts - 1) * t["dt"] - 1e-9, *f.samples)
    series = probe_series(t, oracle.Oracle(t).run(t["n_timesteps"]))[0]
    g = np.load(os.path.join(HERE, "golden", "excitation_test_Ex.npz"))
    v = np.where(np.abs(series) < 1e-30, 0.0, series)
    assert np.linalg.norm(v - g["value"]) / np.linalg.norm(g["value"]) < TOL


def test_file_function_needs_an_opener_and_samples():
    lines = inputs()["excitation_test"]
    with pytest.raises(UnsupportedFeature, match="no file opener"):
        inp.read_inp(lines, materials)
    with pytest.raises(ValueError, match="without samples"):
        inp.read_inp(lines, materials, lambda name: ["# nothing here"][1:])
    with pytest.raises(UnsupportedFeature, match="'noise'"):
        small("Excitation_function_list\n1\n1\nnoise\n1.0\n", BASE.replace(
            "Excitation_function_list\n1\n1\ngaussian\n1.0 1e-9 3e-9\n", ""))


@pytest.mark.gpu
def test_gpu_excitation_function_from_a_file(gpu_lib):
    p = inp.read_inp(inputs()["excitation_test"], materials, data_file)
    t = build_tables(p.spec)
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.run(t["n_timesteps"])
        series = probe_series(t, g.cell_output())[0]
    gold = np.load(os.path.join(HERE, "golden", "excitation_test_Ex.npz"))["value"]
    v = np.where(np.abs(series) < 1e-30, 0.0, series)
    assert np.linalg.norm(v - gold) / np.linalg.norm(gold) < TOL


def test_lenient_reading_leaves_out_only_refused_output_packets():
    lines = inputs()["power_calc"]
    with pytest.raises(UnsupportedFeature, match="rotated rectangle"):
        inp.read_inp(lines, materials)  # strict: the output surface on the rotated rectangle
    p = inp.read_inp_lenient(lines, materials)
    assert p.skipped == ["output_surface_list: an output surface on a rotated rectangle: only zero Euler angles "
                         "are supported"]
    assert p.spec.output_surfaces == [] and len(p.spec.outputs) == 1 and len(p.spec.power_surfaces) == 1
    # geometry and sources are never left out
    with pytest.raises(UnsupportedFeature):
        inp.read_inp_lenient(BASE.splitlines() + ["Cable_list", "0"], materials)


def test_two_corner_blocks_equal_centred_blocks():
    """rectangular_block2 (corners, either order, plus the translation) gives
    the cells and, as a surface, the Huygens box of the centred block with
    the same extent; both builders give the box's triangles inward normals."""
    geo = """Volume_list
2
1
rectangular_block
0.4 0.4 0.6
0 0 0
0.5 0.5 0.5
2
rectangular_block2
0.2 0.2 -0.1   -0.2 -0.2 0.5
0 0 0
0.5 0.5 0.3
Surface_list
2
1
rectangular_block
0.4 0.4 0.6
0 0 0
0.5 0.5 0.5
2
rectangular_block2
-0.2 -0.2 -0.3   0.2 0.2 0.3
0 0 0
0.5 0.5 0.5
Volume_material_list
2
1
PEC
1
1
2
PMC
1
2
"""
    hs = "Huygens_surface\n{n}\n-1\n1\n30.0 20.0\n1.0 0.0\n"
    a = small(geo + hs.format(n=1))
    b = small(geo + hs.format(n=2))
    (_, b1), (_, b2) = a.spec.material_regions
    assert b1 == b2 and (b1.i0, b1.i1, b1.k0, b1.k1) == (4, 7, 3, 8)
    assert a.spec.huygens == b.spec.huygens
