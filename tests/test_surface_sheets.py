"""PEC, PMC and free-space surface materials on internal faces
(connect_normal_to_x.F90:36-52 and the y, z analogues): the connect across
a sheet reflects each side with -1 (PEC) or +1 (PMC), or is the plain
connect (free space).

CPU: the tables, and on the oracle that a sheet across the whole section
lets nothing through while a free-space sheet changes nothing.  GPU: FP64
against the oracle (full and partial sheets, all three axes, with face
outputs on a sheet), FP32 against FP64, batched against solo, and the
rejection of other surface materials."""
import os
import sys

import numpy as np
import pytest

from ggi_tlm_b200 import capi, cases
from ggi_tlm_b200.problem import DFTSurface, OutputPoint, SurfaceSheet, UnsupportedFeature, build_tables, probe_series

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import oracle  # noqa: E402

PROBES = [OutputPoint((12, 12, 19), "Ex"), OutputPoint((12, 12, 20), "Ey"), OutputPoint((12, 12, 10), "Ex"),
          OutputPoint((6, 17, 14), "Ez")]


def spec_with(sheets, steps=80, dft=False):
    spec = cases.pml_point_source(24, pml=4, steps=steps, n_probes=0)
    spec.surface_sheets = sheets
    spec.outputs = list(PROBES)
    if dft:  # face outputs on a sheet's faces
        spec.dft_surfaces = [DFTSurface(1, 13, (8, 16), (8, 16), [1e9, 3e9], "Ey")]
    return spec


FULL_PEC = [SurfaceSheet("PEC", 3, 16, (1, 24), (1, 24))]
PARTIAL = [SurfaceSheet("PEC", 3, 15, (6, 18), (6, 18)), SurfaceSheet("PMC", 1, 13, (8, 16), (8, 16)),
           SurfaceSheet("PEC", 2, 9, (5, 20), (10, 14))]


def oracle_probes(t):
    o = oracle.Oracle(t)
    return probe_series(t, o.run(t["n_timesteps"])), o


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_tables_and_oracle_physics():
    t = build_tables(spec_with(FULL_PEC))
    assert int((t["face_mat"] == 1).sum()) == 24 * 24 and t["n_faces"] == 24 * 24
    base, _ = oracle_probes(build_tables(spec_with([])))
    for kind in ("PEC", "PMC"):
        p, _ = oracle_probes(build_tables(spec_with([SurfaceSheet(kind, 3, 16, (1, 24), (1, 24))])))
        assert not np.any(p[0]) and not np.any(p[1])        # nothing behind a full sheet
        assert np.abs(p[2]).max() > 0 and not np.array_equal(p[2], base[2])  # reflection in front
    pf, _ = oracle_probes(build_tables(spec_with([SurfaceSheet("free", 3, 16, (1, 24), (1, 24))])))
    assert np.array_equal(pf, base)                          # a free-space sheet changes nothing
    with pytest.raises(UnsupportedFeature):
        build_tables(spec_with([SurfaceSheet("thin_layer", 3, 16, (1, 24), (1, 24))]))


@pytest.mark.gpu
def test_gpu_fp64_matches_oracle(gpu_lib):
    for sheets, dft in ((FULL_PEC, False), (PARTIAL, True)):
        t = build_tables(spec_with(sheets, dft=dft))
        want, o = oracle_probes(t)
        with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
            g.run(t["n_timesteps"])
            got = probe_series(t, g.cell_output())
            gd = g.dft() if dft else None
        for a, b in zip(got, want):
            if np.any(b):
                assert rel(a, b) < 1e-10
            else:
                assert not np.any(a)
        if dft:
            assert rel(gd, o.dft()) < 1e-10


@pytest.mark.gpu
def test_gpu_fp32_and_batch_equals_solo(gpu_lib):
    t = build_tables(spec_with(PARTIAL, steps=100))
    res = {}
    for prec in (capi.TLM_PRECISION_FP32, capi.TLM_PRECISION_FP64):
        with capi.GpuMesh(t, precision=prec) as g:
            g.set_variant(1)
            g.run(t["n_timesteps"])
            res[prec] = probe_series(t, g.cell_output())
    for a, b in zip(res[capi.TLM_PRECISION_FP32], res[capi.TLM_PRECISION_FP64]):
        assert rel(a, b) < 1e-3
    other = build_tables(cases.pml_point_source(20, steps=40, pml=3, n_probes=1))
    meshes = [capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP32), capi.GpuMesh(other, precision=capi.TLM_PRECISION_FP32)]
    b = capi.GpuBatch(meshes)
    b.set_variant(1)
    b.run(t["n_timesteps"])
    batched = probe_series(t, meshes[0].cell_output())
    b.close()
    for g in meshes:
        g.close()
    assert np.array_equal(batched, res[capi.TLM_PRECISION_FP32])


@pytest.mark.gpu
def test_gpu_rejects_other_surface_materials(gpu_lib):
    t = build_tables(spec_with(FULL_PEC, steps=10))
    t["face_mat"] = t["face_mat"].copy()
    t["face_mat"][0] = 5  # a surface material type outside PEC, PMC, thin layer and free space (a diode)
    with pytest.raises(capi.TLMError) as e:
        with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
            g.run(1)
    assert "TLM_E_UNSUPPORTED" in str(e.value)
    t["face_mat"][0] = 3  # a thin layer without its thin-layer material
    with pytest.raises(capi.TLMError) as e:
        with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
            g.run(1)
    assert "TLM_E_BADARG" in str(e.value)
