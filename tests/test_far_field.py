"""Far-field surface accumulators (OUTPUT/far_field_surfaces.F90:252-351).

The far-field J, M of a face are dt times the running Fourier sums of n x H
and -(n x E) on that face, which the frequency-output surfaces
(frequency_output_surfaces.F90, pinned separately) also accumulate; the
oracle's far-field sums must agree with dt times its DFT sums of the same
face fields.  The GPU path is checked against the oracle.
"""
import numpy as np
import pytest

from ggi_tlm_b200 import capi
from ggi_tlm_b200.problem import (DFTSurface, ExcitationFunction, FarFieldSurface, OutputPoint, PointExcitation,
                                  ProblemSpec, build_tables, probe_series)

import oracle as O

FREQS = [0.4e9, 1.1e9]


def spec(steps=240, box=True):
    s = ProblemSpec(nx=24, ny=22, nz=20, dl=1e-2, n_timesteps=steps, R=(0.0,) * 6,
                    functions=[ExcitationFunction("gaussian", (1.0, 0.1e-9, 0.4e-9))],
                    point_excitations=[PointExcitation((12, 11, 10), "Ez", 1), PointExcitation((11, 12, 11), "Hx", 1)],
                    outputs=[OutputPoint((15, 12, 10), "Ez")])
    plane = (3, 14, (6, 18), (5, 17))
    s.far_field_surfaces = [FarFieldSurface(FREQS, plane=plane)]
    if box:
        s.far_field_surfaces.append(FarFieldSurface([0.8e9], box=((7, 17), (6, 16), (5, 15))))
        s.far_field_surfaces.append(FarFieldSurface([0.8e9], box=((8, 16), (7, 15), (6, 14)), side=-1))
    s.dft_surfaces = [DFTSurface(axis=3, index=14, r0=(6, 18), r1=(5, 17), frequencies=FREQS, component=c)
                      for c in ("Ex", "Ey", "Jx", "Jy", "Jz")]
    return s


def test_far_field_tables():
    t = build_tables(spec())
    n_plane = 13 * 13
    n_box = 2 * (11 * 11 + 11 * 11 + 11 * 11)
    n_box2 = 2 * (9 * 9 * 3)
    assert t["n_ff"] == 4
    assert list(np.diff(t["ff_face_ptr"])) == [n_plane, n_plane, n_box, n_box2]
    # side 1 box faces sit on the outside cells: their codes are max faces on the min planes
    codes = t["ff_face_code"][2 * n_plane:2 * n_plane + n_box]
    assert sorted(set(codes.tolist())) == [1, 2, 3, 4, 5, 6]


def test_oracle_far_field_is_dt_times_the_face_dft():
    t = build_tables(spec(box=False))
    o = O.Oracle(t)
    o.run(t["n_timesteps"])
    ff = o.far_field()                    # [entries, 6]
    dft = o.dft()                          # [(component, frequency, face), 2]
    nf = 13 * 13
    d = (dft[:, 0] + 1j * dft[:, 1]).reshape(5, 2, nf)   # Ex, Ey, Jx, Jy, Jz
    dt = t["dt"]
    for fi in range(2):
        J = ff[fi * nf:(fi + 1) * nf, :3]
        M = ff[fi * nf:(fi + 1) * nf, 3:]
        # z-plane min faces: n = +z, so n x E = (-Ey, Ex, 0) and M = -(n x E) = (Ey, -Ex, 0)
        for c in range(3):
            np.testing.assert_allclose(J[:, c], dt * d[2 + c, fi], rtol=1e-12, atol=1e-12 * np.abs(J).max())
        np.testing.assert_allclose(M[:, 0], dt * d[1, fi], rtol=1e-12, atol=1e-12 * np.abs(M).max())
        np.testing.assert_allclose(M[:, 1], -dt * d[0, fi], rtol=1e-12, atol=1e-12 * np.abs(M).max())
        assert np.abs(M[:, 2]).max() == 0.0
    assert np.abs(ff).max() > 0


@pytest.mark.gpu
def test_gpu_far_field_matches_oracle(gpu_lib):
    t = build_tables(spec())
    o = O.Oracle(t)
    po = probe_series(t, o.run(t["n_timesteps"]))
    fo = o.far_field()
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.run(100)
        g.run(t["n_timesteps"] - 100)
        fg = g.far_field()
        pg = probe_series(t, g.cell_output())
    assert np.linalg.norm(pg - po) <= 1e-10 * np.linalg.norm(po)
    assert np.linalg.norm(fg - fo) <= 1e-10 * np.linalg.norm(fo)
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP32) as g:
        g.run(t["n_timesteps"])
        f32 = g.far_field()
    assert np.linalg.norm(f32 - fo) <= 1e-4 * np.linalg.norm(fo)


@pytest.mark.gpu
def test_gpu_far_field_in_a_batch_equals_solo(gpu_lib):
    tabs = [build_tables(spec(150)), build_tables(spec(120, box=False))]
    solo = []
    for t in tabs:
        with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
            g.set_variant(1)
            g.run(t["n_timesteps"])
            solo.append(g.far_field())
    meshes = [capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) for t in tabs]
    with capi.GpuBatch(meshes) as b:
        b.set_variant(1)
        b.run(1000)
    for g, ff in zip(meshes, solo):
        assert np.array_equal(g.far_field(), ff)
        g.close()
