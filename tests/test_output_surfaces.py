"""Time-domain output surfaces (OUTPUT/output_surfaces.F90:601-760): on each
output step every face of the surface records E, H, J = n x H or a
magnitude from face_output_field after connect.

CPU: the tables and the oracle restatement's own identities (J = n x H
against the H surfaces, magnitudes against their components).  GPU: FP64
against the oracle, FP32 against FP64, batched against solo, a partial
run, and argument errors."""
import os
import sys

import numpy as np
import pytest

from ggi_tlm_b200 import capi, cases
from ggi_tlm_b200.problem import OutputSurface, build_tables

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import oracle  # noqa: E402

PLANE = (3, 12, (6, 18), (6, 18))  # z-normal patch across the plane wave
BOX = ((8, 16), (8, 16), (8, 16))


def spec_with_surfaces(steps=60):
    spec = cases.pml_spheres(n=24, pml=4, n_spheres=3, steps=steps, n_probes=4, n_freq=3, dft_size=6, rmin=2.0,
                             rmax=3.5)
    spec.output_surfaces = [
        OutputSurface("Ey", plane=PLANE, first_step=3, interval=4),              # gated steps
        OutputSurface("Jm", box=BOX, side=-1, last_step=50),                    # flipped faces, stops early
        OutputSurface("Hm", box=BOX),                                           # scale for the next one
        OutputSurface("Jy", box=BOX, both_sides=True, interval=2),              # both sides: ~ round-off
        OutputSurface("Em", plane=PLANE),
        OutputSurface("Hx", plane=PLANE),
        OutputSurface("Hy", plane=PLANE),
        OutputSurface("Jx", plane=PLANE),
        OutputSurface("Jm", plane=PLANE),
    ]
    return spec


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_tables():
    spec = spec_with_surfaces()
    t = build_tables(spec)
    assert t["n_osurf"] == 9
    shapes = capi.output_surface_shapes(t)
    assert shapes[0] == (15, 13 * 13)          # steps 3, 7, ..., 59
    assert shapes[1][0] == 50 and shapes[3][0] == 30
    assert shapes[1][1] == shapes[2][1] == 6 * 9 * 9  # six 9x9 faces of the box
    ptr, codes = t["osurf_face_ptr"], t["osurf_face_code"]
    box_flipped, box = codes[ptr[1]:ptr[2]], codes[ptr[2]:ptr[3]]
    assert np.array_equal(np.where(box <= 3, box + 3, box - 3), box_flipped)  # side -1 samples the other side
    assert set(t["osurf_comp"]) == {2, 15, 14, 8, 13, 4, 5, 7}
    with pytest.raises(ValueError):
        bad = spec_with_surfaces()
        bad.output_surfaces[0].component = "Mx"
        build_tables(bad)


def test_oracle_identities():
    t = build_tables(spec_with_surfaces())
    r = oracle.output_surfaces(t)
    ey, em, hx, hy, jx, jm = r[0], r[4], r[5], r[6], r[7], r[8]
    assert np.abs(ey).max() > 0 and np.abs(hx).max() > 0
    # the plane's faces are min z faces (n = +z): Jx = -Hy, |J| = sqrt(Hx^2 + Hy^2)
    assert np.array_equal(jx, -hy)
    assert np.allclose(jm, np.sqrt(hx ** 2 + hy ** 2), rtol=1e-14, atol=0)
    assert np.all(em >= 0) and np.all(em[2::4] >= np.abs(ey) * (1 - 1e-15))  # Ey's steps 3, 7, ... are rows 2, 6, ...
    # both sides of interior faces carry the same H, so J is round-off against the one-sided |H|
    assert np.abs(r[3]).max() <= 1e-10 * np.abs(r[2]).max()


@pytest.mark.gpu
def test_gpu_fp64_matches_oracle(gpu_lib):
    t = build_tables(spec_with_surfaces())
    want = oracle.output_surfaces(t)
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.run(t["n_timesteps"])
        got = g.output_surfaces()
    for k, (a, b) in enumerate(zip(got, want)):
        assert a.shape == b.shape
        if k == 3:  # both-sides J: round-off, judged against the one-sided |H| on the same faces
            assert np.abs(a - b).max() <= 1e-10 * np.abs(want[2]).max()
        else:
            assert rel(a, b) < 1e-10, k


@pytest.mark.gpu
def test_gpu_fp32_batch_and_partial_run(gpu_lib):
    t = build_tables(spec_with_surfaces(steps=80))
    res = {}
    for prec in (capi.TLM_PRECISION_FP32, capi.TLM_PRECISION_FP64):
        with capi.GpuMesh(t, precision=prec) as g:
            g.set_variant(1)
            g.run(t["n_timesteps"])
            res[prec] = g.output_surfaces()
    for k in (0, 1, 2, 4, 5, 8):
        assert rel(res[capi.TLM_PRECISION_FP32][k], res[capi.TLM_PRECISION_FP64][k]) < 1e-3, k
    # in a batch with another mesh: bit-identical to solo
    other = build_tables(cases.pml_point_source(20, steps=50, pml=3, n_probes=1))
    meshes = [capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP32), capi.GpuMesh(other, precision=capi.TLM_PRECISION_FP32)]
    b = capi.GpuBatch(meshes)
    b.set_variant(1)
    b.run(t["n_timesteps"])
    batched = meshes[0].output_surfaces()
    b.close()
    for g in meshes:
        g.close()
    for a, c in zip(batched, res[capi.TLM_PRECISION_FP32]):
        assert np.array_equal(a, c)
    # after 30 of 80 steps: the rows of the steps run so far, zeros after
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP32) as g:
        g.set_variant(1)
        g.run(30)
        part = g.output_surfaces()
    ey_full, ey_part = res[capi.TLM_PRECISION_FP32][0], part[0]
    n_done = len(range(3, 31, 4))
    assert np.array_equal(ey_part[:n_done], ey_full[:n_done])
    assert not np.any(ey_part[n_done:])


@pytest.mark.gpu
def test_gpu_rejects_bad_surface_arguments(gpu_lib):
    for key, value in (("osurf_comp", 10), ("osurf_face_code", 7), ("osurf_interval", 0), ("osurf_both", 2)):
        t = build_tables(spec_with_surfaces(steps=10))
        t[key] = t[key].copy()
        t[key][0] = value
        with pytest.raises(capi.TLMError) as e:
            with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
                g.run(1)
        assert "TLM_E_BADARG" in str(e.value)
