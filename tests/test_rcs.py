"""The RCS surface's time-domain far field (OUTPUT/RCS_surfaces.F90:159-560):
every step each face adds its far-field contribution to the time bin that
its delay along K and the step's time select.

CPU: the far-field array size and offset (initialise_rcs_surfaces), the
monotone bin order the GPU kernel relies on, and the oracle restatement.
GPU: FP64 against the oracle (the bins must match exactly for this to
hold), FP32 against FP64, batched against solo, and argument errors."""
import math
import os
import sys

import numpy as np
import pytest

from ggi_tlm_b200 import capi, cases
from ggi_tlm_b200.problem import C0, RCSSurface, build_tables

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import oracle  # noqa: E402


def spec_with_rcs(steps=80, theta=30.0, phi=45.0, **kw):
    spec = cases.pml_spheres(n=24, pml=4, n_spheres=3, steps=steps, n_probes=4, n_freq=3, dft_size=6, rmin=2.0,
                             rmax=3.5)
    spec.rcs_surface = RCSSurface(theta, phi, **(kw or {"box": ((8, 16), (8, 16), (8, 16))}))
    return spec


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_tables_and_bin_order():
    t = build_tables(spec_with_rcs())
    dist = t["rcs_face_dist"]
    assert len(dist) == 6 * 9 * 9
    dl, dt = t["dl"], t["dt"]
    dmin, dmax = dist.min(), dist.max()
    distance = ((dmax - dmin) / C0 + t["n_timesteps"] * dt) * C0
    assert t["rcs_points"] == int(2 * distance / dl + 2)
    assert t["rcs_offset"] == int(2 * dmin / dl - 1)
    assert abs(t["rcs_theta"] - math.radians(30.0)) < 1e-15
    # along K.x ascending the bins never increase, so each bin is one run of faces
    order = np.argsort(dist, kind="stable")
    for step in (1, 17, 40, 80):
        tc0 = ((step - 1) * dt + dt / 2.0) * C0
        pts = [int(2.0 * (-float(dist[f]) + tc0) / dl) - int(t["rcs_offset"]) for f in order]
        assert all(a >= b for a, b in zip(pts, pts[1:]))
    # a plane normal to x along theta = 90, phi = 0: every face at one delay
    tp = build_tables(spec_with_rcs(theta=90.0, phi=0.0, plane=(1, 12, (6, 18), (6, 18))))
    assert np.ptp(tp["rcs_face_dist"]) < 1e-12


def test_oracle_far_field():
    t = build_tables(spec_with_rcs())
    a = oracle.rcs(t)
    assert a.shape == (4, t["rcs_points"])
    assert np.count_nonzero(a[0]) > 10 and np.abs(a).max() > 0


@pytest.mark.gpu
def test_gpu_fp64_matches_oracle(gpu_lib):
    for kw in ({}, {"theta": 90.0, "phi": 0.0, "plane": (1, 12, (6, 18), (6, 18))}):
        t = build_tables(spec_with_rcs(**kw))
        want = oracle.rcs(t)
        with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
            g.run(t["n_timesteps"])
            got = g.rcs()
        for k in range(4):
            assert rel(got[k], want[k]) < 1e-10, (kw, k)


@pytest.mark.gpu
def test_gpu_fp32_and_batch_equals_solo(gpu_lib):
    t = build_tables(spec_with_rcs(steps=100))
    res = {}
    for prec in (capi.TLM_PRECISION_FP32, capi.TLM_PRECISION_FP64):
        with capi.GpuMesh(t, precision=prec) as g:
            g.set_variant(1)
            g.run(t["n_timesteps"])
            res[prec] = g.rcs()
    for k in range(4):
        assert rel(res[capi.TLM_PRECISION_FP32][k], res[capi.TLM_PRECISION_FP64][k]) < 1e-3
    other = build_tables(cases.pml_point_source(20, steps=40, pml=3, n_probes=1))
    meshes = [capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP32), capi.GpuMesh(other, precision=capi.TLM_PRECISION_FP32)]
    b = capi.GpuBatch(meshes)
    b.set_variant(1)
    b.run(t["n_timesteps"])
    batched = meshes[0].rcs()
    b.close()
    for g in meshes:
        g.close()
    assert np.array_equal(batched, res[capi.TLM_PRECISION_FP32])


@pytest.mark.gpu
def test_gpu_rejects_bad_rcs_arguments(gpu_lib):
    for key, value in (("rcs_face_code", 0), ("rcs_face_out", 10 ** 6)):
        t = build_tables(spec_with_rcs(steps=10))
        t[key] = t[key].copy()
        t[key][0] = value
        with pytest.raises(capi.TLMError) as e:
            with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
                g.run(1)
        assert "TLM_E_BADARG" in str(e.value)
