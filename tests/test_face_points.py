"""Point sources and output points on cell faces.

Face sources (EXCITATION/excitation_points.F90:286-323) add the function's
value_face on both sides of the face, hard or soft per component; connect
applies them (TLM_SOLVER/connect_normal_to_{x,y,z}.F90).  Face output points
(OUTPUT/output_points.F90:255-444) record one side of face_output_field after
connect.  The oracle restates both; the GPU path is checked against it.
"""
import numpy as np
import pytest

from ggi_tlm_b200 import capi
from ggi_tlm_b200.problem import (ExcitationFunction, HuygensPlane, OutputPoint, PointExcitation, ProblemSpec,
                                  UnsupportedFeature, build_tables, probe_series)

import oracle as O

STEPS = 300


def spec(steps=STEPS, huygens=False):
    s = ProblemSpec(
        nx=20, ny=18, nz=16, dl=5e-3, n_timesteps=steps, R=(-1.0,) * 6,
        functions=[ExcitationFunction("gaussian", (1.0, 0.05e-9, 0.2e-9)),
                   ExcitationFunction("differential_gaussian", (1.0, 0.05e-9, 0.2e-9))],
        point_excitations=[PointExcitation((10, 9, 8), "Ey", 1, face="xmax"),
                           PointExcitation((5, 5, 5), "Jz", 2, face="zmin"),
                           PointExcitation((14, 12, 10), "Hx", 1, source_type=0, face="ymax"),
                           PointExcitation((6, 7, 8), "Mx", 2, face="ymin"),
                           PointExcitation((6, 7, 8), "Ez", 1, face="ymin"),
                           PointExcitation((15, 4, 12), "Ez", 1)],
        outputs=[OutputPoint((12, 9, 8), "Ey"), OutputPoint((10, 9, 8), "Ey", face="xmax"),
                 OutputPoint((11, 9, 8), "Hz", face="xmin"), OutputPoint((7, 7, 7), "Ex", face="zmax"),
                 OutputPoint((3, 14, 9), "Hy", face="xmin"), OutputPoint((6, 7, 8), "Hx", face="ymin"),
                 OutputPoint((6, 6, 8), "Hx", face="ymax")])
    if huygens:  # a Huygens plane sharing faces with a point source
        s.huygens = HuygensPlane(axis=2, index=6, r0=(3, 17), r1=(3, 14), function=1, ktheta=90.0, kphi=90.0,
                                 etheta=1.0, ephi=0.0)
    return s


def test_face_tables():
    assert build_tables(spec(huygens=True))["hs_n"] == 15 * 12
    t = build_tables(spec())
    assert t["n_face_points"] == 5 and t["n_face_probes"] == 6 and t["n_exc_cells"] == 1
    # the xmax face of cell (10,9,8) is the xmin face of cell (11,9,8): one output face, two sides
    assert t["fprobe_face"][0] == t["fprobe_face"][1] and list(t["fprobe_side"][:2]) == [2, 1]
    # two sources on one face share its excitation face number
    assert t["fpt_face"][3] == t["fpt_face"][4]
    # sides ymin of (6,7,8) and ymax of (6,6,8) are the same face
    assert t["fprobe_face"][4] == t["fprobe_face"][5] and list(t["fprobe_side"][4:]) == [1, 2]


def test_face_table_errors():
    s = spec()
    s.point_excitations.append(PointExcitation((1, 5, 5), "Ey", 1, face="xmin"))
    with pytest.raises(UnsupportedFeature):
        build_tables(s)  # a face of the outer boundary
    s = spec()
    s.outputs.append(OutputPoint((5, 5, 5), "Jx", face="zmin"))
    with pytest.raises(ValueError):
        build_tables(s)
    s = spec()
    s.point_excitations.append(PointExcitation((5, 5, 5), "Mx", 1))
    with pytest.raises(ValueError):
        build_tables(s)


def test_oracle_face_sources_drive_the_face_probes():
    t = build_tables(spec())
    o = O.Oracle(t)
    o.run(STEPS)
    fp = o.face_probes()
    assert fp.shape == (6, STEPS) and np.all(np.abs(fp).max(axis=1) > 0)
    # a hard Hx source on its face forces H there: the probe on that face follows the function
    # only through the connect; with the source removed the series changes
    s = spec()
    s.point_excitations = s.point_excitations[:2]
    t2 = build_tables(s)
    o2 = O.Oracle(t2)
    o2.run(STEPS)
    assert np.abs(o2.face_probes()[3] - fp[3]).max() > 1e-3 * np.abs(fp[3]).max()


@pytest.mark.gpu
@pytest.mark.parametrize("huygens", [False, True])
def test_gpu_face_points_match_oracle(gpu_lib, huygens):
    t = build_tables(spec(huygens=huygens))
    o = O.Oracle(t)
    po = probe_series(t, o.run(STEPS))
    fo = o.face_probes()
    lo = o.links()
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.run(77)
        g.run(STEPS - 77)
        pg = probe_series(t, g.cell_output())
        fg = g.face_output()
        lg = g.links()
    for i in range(fo.shape[0]):
        assert np.linalg.norm(fg[i] - fo[i]) <= 1e-10 * np.linalg.norm(fo[i])
    assert np.linalg.norm(pg[0] - po[0]) <= 1e-10 * np.linalg.norm(po[0])
    assert np.abs(lg - lo).max() <= 1e-10 * np.abs(lo).max()
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP32) as g:
        g.run(STEPS)
        f32 = g.face_output()
    for i in range(fo.shape[0]):
        assert np.linalg.norm(f32[i] - fo[i]) <= 1e-4 * np.linalg.norm(fo[i])


@pytest.mark.gpu
def test_gpu_face_points_in_a_batch_equal_solo(gpu_lib):
    tabs = [build_tables(spec(200)), build_tables(spec(150, huygens=True))]
    solo = []
    for t in tabs:
        with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
            g.set_variant(1)
            g.run(t["n_timesteps"])
            solo.append((g.cell_output(), g.face_output()))
    meshes = [capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) for t in tabs]
    with capi.GpuBatch(meshes) as b:
        b.set_variant(1)
        b.run(1000)
    for g, (co, fo) in zip(meshes, solo):
        assert np.array_equal(g.cell_output(), co) and np.array_equal(g.face_output(), fo)
        g.close()


@pytest.mark.gpu
def test_gpu_face_point_argument_errors(gpu_lib):
    t = dict(build_tables(spec(10)))
    t["fpt_comp"] = np.array(t["fpt_comp"]).copy()
    t["fpt_comp"][0] = 13
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        with pytest.raises(capi.TLMError) as e:
            g.run(1)
        assert e.value.code == capi.TLM_E_BADARG
