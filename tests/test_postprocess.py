"""Host-side result files from the device accumulators
(ggi_tlm_b200/postprocess.py): the far-field pattern
(far_field_surfaces.F90:370-712) and SAR (SAR_volumes.F90:334-622).

The SAR file's list-directed lines are checked against the reference's
SAR_TEST golden file (tests/golden/result_text.npz); the far-field transform
against the radiation pattern of a small dipole (|E_theta| ~ sin theta,
E_phi ~ 0) computed from the oracle's far-field accumulators; SAR against
its definition on the oracle's accumulators.  GPU: the library's
accumulators give the oracle's files."""
import os
import sys

import numpy as np
import pytest

from ggi_tlm_b200 import postprocess as pp
from ggi_tlm_b200.problem import (Block, FarFieldSurface, PointExcitation, SARVolume, VolumeMaterial, build_tables)
from ggi_tlm_b200 import cases

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import oracle  # noqa: E402


def test_sar_lines_match_the_reference_file():
    lines = [str(x) for x in np.load(os.path.join(HERE, "golden", "result_text.npz"))["sar_test"]]
    assert len(lines) == 2
    for k, line in enumerate(lines, start=1):
        f, n, v = line.split()
        assert int(n) == k
        assert pp.sar_line(float(f), k, float(v)) == line


def test_list_directed_reals():
    assert pp._ld_real(0.5) == "0.50000000000000000".rjust(21) + " " * 5
    assert pp._ld_real(-12.25) == "-12.250000000000000".rjust(21) + " " * 5
    assert pp._ld_real(1e17) == "1.0000000000000000E+017".rjust(26)
    assert pp._ld_real(0.05) == "5.0000000000000003E-002".rjust(26)
    assert pp._ld_real(0.0) == "0.0000000000000000".rjust(21) + " " * 5


def test_face_points():
    o, dl = (-1.0, 0.0, 2.0), 0.5
    assert pp.face_point(o, dl, (1, 1, 1), 7) == (-0.75, 0.25, 2.25)
    assert pp.face_point(o, dl, (1, 1, 1), 1) == (-1.0, 0.25, 2.25)
    assert pp.face_point(o, dl, (1, 1, 1), 6) == (-0.75, 0.25, 2.5)


def dipole_spec(n=32, steps=400):
    """A PML box with a soft Ez point source at its centre and a closed
    far-field box around it, 300 MHz (wavelength 100 cells)."""
    s = cases.pml_point_source(n, pml=6, steps=steps, dl=0.01, n_probes=0)
    c = (n + 1) // 2
    s.point_excitations = [PointExcitation((c, c, c), "Ez", 1)]
    s.far_field_surfaces = [FarFieldSurface([3e8], box=((10, n - 9), (10, n - 9), (10, n - 9)))]
    return s


POST = dict(frequency=3e8, theta=(0.0, 180.0, 10.0), phi=(0.0, 90.0, 45.0), dim=3)


def test_small_dipole_far_field_pattern():
    s = dipole_spec()
    t = build_tables(s)
    o = oracle.Oracle(t)
    o.run(t["n_timesteps"])
    acc = o.far_field()
    o.close()
    th, ph, et, ep = pp.far_field_pattern(acc, pp.far_field_face_points(s, t)[0], dl=s.dl, **POST)
    assert len(th) == 19 * 3
    peak = et.max()
    assert peak > 0
    ok = (th > np.radians(15)) & (th < np.radians(165))
    np.testing.assert_allclose(et[ok] / peak, np.sin(th[ok]), atol=0.02)
    assert ep.max() < 1e-2 * peak
    lines = pp.far_field_lines(th, ph, et, ep, 19, 3, t["dt"])
    assert lines[0] == "#     19     3" + pp._es(1.0 / t["dt"], 16, 6) and len(lines) == 1 + 57
    assert lines[1].split()[:2] == ["0.000000E+00", "0.000000E+00"]


def sar_spec():
    s = cases.pml_point_source(24, pml=5, steps=300, dl=0.01, n_probes=0)
    s.materials = [VolumeMaterial.dielectric(4.0, 0.5)]
    s.material_regions = [(1, Block(10, 15, 10, 15, 14, 17))]
    s.sar_volumes = [SARVolume(Block(10, 15, 10, 15, 14, 17), [3e8])]
    return s


def test_sar_value_is_its_definition():
    s = sar_spec()
    t = build_tables(s)
    o = oracle.Oracle(t)
    co = o.run(t["n_timesteps"])
    o.close()
    acc = oracle.sar_volumes(t, co)
    (f, n, v), = pp.sar_values(s, t, acc, [1000.0])
    e2 = 0.5 * np.sum(np.abs(acc) ** 2)
    assert (f, n) == (3e8, 1) and v > 0
    assert v == pytest.approx(e2 * 0.5 * s.dl ** 3 / (s.dl ** 3 * 1000.0 * acc.shape[0]), rel=1e-12)
    bad = sar_spec()
    bad.materials = [VolumeMaterial.debye(2.0, [4.0], [1e-10])]
    with pytest.raises(ValueError, match="dispersive dielectric"):
        pp.sar_values(bad, t, acc, [1000.0])


@pytest.mark.gpu
def test_gpu_far_field_and_sar_files_match_the_oracle(gpu_lib, tmp_path):
    from ggi_tlm_b200 import capi

    s = dipole_spec(steps=300)
    s.materials = [VolumeMaterial.dielectric(4.0, 0.5)]
    s.material_regions = [(1, Block(12, 14, 12, 14, 18, 20))]
    s.sar_volumes = [SARVolume(Block(12, 14, 12, 14, 18, 20), [3e8])]
    t = build_tables(s)
    o = oracle.Oracle(t)
    co = o.run(t["n_timesteps"])
    ff_o, sar_o = o.far_field(), oracle.sar_volumes(t, co)
    o.close()
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.run(t["n_timesteps"])
        ff_g, sar_g = g.far_field(), g.sar_volumes()
    pts = pp.far_field_face_points(s, t)[0]
    a = pp.far_field_pattern(ff_g, pts, dl=s.dl, **POST)
    b = pp.far_field_pattern(ff_o, pts, dl=s.dl, **POST)
    for x, y in zip(a, b):
        assert np.linalg.norm(x - y) <= 1e-10 * np.linalg.norm(y)
    (_, _, vg), = pp.sar_values(s, t, sar_g, [1000.0])
    (_, _, vo), = pp.sar_values(s, t, sar_o, [1000.0])
    assert vg == pytest.approx(vo, rel=1e-10)


def plate_input(drop=("surface_material_list",)):
    """RCS_PEC_PLATE_ROUGH_SURFACE's plate.inp without the packets named
    (its plate has a random rough surface, which is not reproducible)."""
    sys.path.insert(0, HERE)
    import test_inp as T
    from ggi_tlm_b200 import inp

    keep, skip = [], False
    for ln in T.inputs()["rcs_plate"]:
        key = ln.strip().split()[0].lower() if ln.strip() else ""
        if key and not ln[:1].isspace() and key[0].isalpha() and key in inp.PACKETS:
            skip = key in drop
        if not skip:
            keep.append(ln)
    return inp.read_inp(keep, T.materials)


def test_rcs_files_match_the_reference_columns():
    """The RCS files of the reference's plate case: the far-field array has
    the reference's length (simulation time from the problem file), the
    .rcs.tout time column and the .rcs.fout frequency and incident-field
    columns are the golden file's, line for line (the scattered-field
    columns depend on the rough plate and are not compared)."""
    p = plate_input()
    t = build_tables(p.spec)
    g = np.load(os.path.join(HERE, "golden", "result_text.npz"))
    fo, to = [str(x) for x in g["rcs_plate_fout"]], [str(x) for x in g["rcs_plate_tout"]]
    assert int(t["rcs_points"]) == len(to)
    tout, fout = pp.rcs_lines(t, np.zeros((4, int(t["rcs_points"]))), *p.post["rcs"], int(t["hs_fn"]))
    assert len(fout) == len(fo) and len(tout) == len(to)
    assert [a[:24] for a in tout] == [b[:24] for b in to]
    assert [(a[:14], a[42:56]) for a in fout] == [(b[:14], b[42:56]) for b in fo]
    assert all(a.endswith("-0.100000E+04") for a in fout)  # no scattered field: RCS -1000


@pytest.mark.gpu
def test_gpu_pec_plate_rcs_follows_physical_optics(gpu_lib):
    """The plate case with a smooth 25 x 25 cm PEC plate (the reference's
    plate sits on z = 0, half a cell off the mesh planes; here on the plane
    below): the monostatic RCS from the GPU's far field is within 1.5 dB of
    physical optics, 4 pi A^2 / lambda^2, from 1.5 to 3 GHz."""
    from ggi_tlm_b200 import capi
    from ggi_tlm_b200.problem import SurfaceSheet

    p = plate_input()
    p.spec.surface_sheets = [SurfaceSheet("PEC", 3, 20, (9, 33), (9, 33))]
    t = build_tables(p.spec)
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.run(t["n_timesteps"])
        far = g.rcs()
    _, fout = pp.rcs_lines(t, far, *p.post["rcs"], int(t["hs_fn"]))
    area = 0.25 ** 2
    for line in fout:
        f, rcs = float(line[:14]), float(line[56:70])
        if 1.5e9 <= f <= 3e9:
            po = 10.0 * np.log10(4.0 * np.pi * area ** 2 / (299792458.0 / f) ** 2)
            assert abs(rcs - po) < 1.5, (f, rcs, po)


def helix_spec():
    """HELIX_ANTENNA read with its mesh file, cables left out."""
    sys.path.insert(0, HERE)
    import test_inp as T
    import test_meshfile as M
    from ggi_tlm_b200 import inp, meshfile

    m = meshfile.read_mesh(M.helix_mesh_lines())
    return inp.read_inp_lenient(M.without_cables(M.helix_inp_lines()), T.materials, mesh_file=m).spec


def test_surface_field_file_matches_the_reference_template():
    """HELIX_ANTENNA's .surface_field.tout: the header and the template of
    its output surface (1764 faces of the mesh file's surface, 10 frames)
    line for line; the first data frame's framing lines (its values need
    the cable model, which is out of scope)."""
    gold = [str(x) for x in np.load(os.path.join(HERE, "golden", "result_text.npz"))["helix_surface_field"]]
    s = helix_spec()
    t = build_tables(s)
    (surf,) = s.output_surfaces
    n_frames = len(pp._output_steps(surf.first_step, surf.last_step, surf.interval, int(t["n_timesteps"])))
    vals = [np.zeros((n_frames, len(surf.faces())))]
    lines = pp.surface_field_lines(s, t, vals)
    end = gold.index("# END SURFACE FIELD FILE TEMPLATE, OUTPUT SURFACE NUMBER:    1")
    assert lines[:end + 1] == gold[:end + 1]
    frame = gold[end + 1:]
    mine = lines[end + 1:end + 1 + len(frame)]
    assert [a for a in mine if a.startswith("#") or not a.strip().startswith(("0.", "-0."))] == \
        [a for a in frame if a.startswith("#") or not a.strip().startswith(("0.", "-0."))]
    assert len(mine) == len(frame)


def test_volume_field_file_layout():
    """A field output volume's .volume_field.tout: 24 corner points and six
    faces a cell in output_volumes.F90's order, one frame per output step,
    each cell's value written six times."""
    s = cases.pml_point_source(12, pml=2, steps=7, dl=0.5, n_probes=0)
    from ggi_tlm_b200.problem import OutputVolume
    s.origin = (1.0, -2.0, 0.5)
    s.output_volumes = [OutputVolume(Block(3, 4, 5, 5, 6, 6), "Ez", kind="field", first_step=2, interval=3)]
    t = build_tables(s)
    vals = [np.arange(2 * 2, dtype=float).reshape(2, 2) + 0.5]  # steps 2 and 5, two cells
    lines = pp.volume_field_lines(s, t, vals)
    assert lines[:2] == ["# NUMBER OF OUTPUT VOLUMES", "           1"]
    assert lines[3:9] == ["# Number of points:", "        48", "# Number of faces:", "        12",
                          "# Number of frames:", "         2"]
    # first cell (3, 5, 6): corner 1 = origin + (cell - 1) dl, corner 7 = origin + cell dl
    assert lines[9] == pp.fortran_e(2.0, 14, 5) + pp.fortran_e(0.0, 14, 5) + pp.fortran_e(3.0, 14, 5)
    assert lines[9 + 6] == pp.fortran_e(2.5, 14, 5) + pp.fortran_e(0.5, 14, 5) + pp.fortran_e(3.5, 14, 5)
    assert lines[9 + 48] == "  4           0           1           2           3"
    start = lines.index("# START OF VOLUME FIELD OUTPUT DATA")
    assert lines[start + 1:start + 8] == ["# OUTPUT VOLUME NUMBER", "           1", "# FRAME NUMBER", "           1",
                                          "# NUMBER OF cellS", "          12", "# volume FIELD DATA"]
    assert lines[start + 8:start + 20] == [pp.fortran_e(0.5, 14, 5)] * 6 + [pp.fortran_e(1.5, 14, 5)] * 6
    assert lines.count("# START OF VOLUME FIELD OUTPUT DATA") == 2
