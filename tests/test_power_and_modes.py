"""Frequency-domain power surfaces (OUTPUT/frequency_domain_power_surfaces.F90
:287-420) and mode outputs (OUTPUT/output_modes.F90:546-620), both read from
face_output_field after connect every step.

CPU: the tables and the oracle restatements' own identities.  GPU: FP64
against the oracle, FP32 against FP64, batched against solo, and argument
errors."""
import math
import os
import sys

import numpy as np
import pytest

from ggi_tlm_b200 import capi, cases
from ggi_tlm_b200.problem import DFTSurface, ModeOutput, PowerSurface, build_tables

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import oracle  # noqa: E402

PLANE = (3, 12, (6, 18), (6, 18))


def profile(i, j, k):
    return math.sin(math.pi * (i - 5) / 14.0) * math.cos(math.pi * (j - 12) / 28.0)


def spec_with_outputs(steps=70):
    spec = cases.pml_spheres(n=24, pml=4, n_spheres=3, steps=steps, n_probes=4, n_freq=3, dft_size=6, rmin=2.0,
                             rmax=3.5)
    spec.power_surfaces = [PowerSurface([1e9, 3e9], box=((8, 16), (8, 16), (8, 16))),
                           PowerSurface([2e9], plane=PLANE, side=-1)]
    spec.mode_outputs = [ModeOutput("Ey", PLANE, profile), ModeOutput("Hx", PLANE, profile),
                         ModeOutput("Ez", PLANE, profile)]  # Ez is zero here: recorded as 0
    return spec


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_tables_and_oracle_identities():
    spec = spec_with_outputs()
    t = build_tables(spec)
    assert t["n_ps"] == 3 and list(t["ps_face_ptr"]) == [0, 486, 972, 1141]
    assert t["n_modes"] == 3 and list(t["mode_face_ptr"]) == [0, 169, 338, 507]
    p = oracle.power_surfaces(t)
    # the plane's E1 (Ex on a z face) against a DFT surface of Ex on the same faces
    ref = spec_with_outputs()
    ref.power_surfaces, ref.mode_outputs = [], []
    ref.dft_surfaces = [DFTSurface(3, 12, (6, 18), (6, 18), [2e9], "Ex")]
    tr = build_tables(ref)
    o = oracle.Oracle(tr)
    o.run(tr["n_timesteps"])
    d = o.dft()
    dft = d[:, 0] + 1j * d[:, 1]
    plane = p[972:1141]
    assert np.abs(plane[:, 0]).max() > 0
    # side -1 samples the max side of the z-1 faces, i.e. the same faces' other side: equal E tangential
    assert rel(plane[:, 0], dft) < 1e-12
    m = oracle.mode_outputs(t)
    assert m.shape == (3, 70) and np.abs(m[0]).max() > 0 and not np.any(m[2])


@pytest.mark.gpu
def test_gpu_fp64_matches_oracle(gpu_lib):
    t = build_tables(spec_with_outputs())
    wp, wm = oracle.power_surfaces(t), oracle.mode_outputs(t)
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.run(t["n_timesteps"])
        gp, gm = g.power_surfaces(), g.mode_outputs()
    ptr = t["ps_face_ptr"]
    for k in range(t["n_ps"]):
        assert rel(gp[ptr[k]:ptr[k + 1]], wp[ptr[k]:ptr[k + 1]]) < 1e-10, k
    for k in range(2):
        assert rel(gm[k], wm[k]) < 1e-10, k
    assert not np.any(gm[2])


@pytest.mark.gpu
def test_gpu_fp32_and_batch_equals_solo(gpu_lib):
    t = build_tables(spec_with_outputs(steps=90))
    res = {}
    for prec in (capi.TLM_PRECISION_FP32, capi.TLM_PRECISION_FP64):
        with capi.GpuMesh(t, precision=prec) as g:
            g.set_variant(1)
            g.run(t["n_timesteps"])
            res[prec] = (g.power_surfaces(), g.mode_outputs())
    assert rel(res[capi.TLM_PRECISION_FP32][0], res[capi.TLM_PRECISION_FP64][0]) < 1e-3
    assert rel(res[capi.TLM_PRECISION_FP32][1][:2], res[capi.TLM_PRECISION_FP64][1][:2]) < 1e-3
    other = build_tables(cases.pml_point_source(20, steps=40, pml=3, n_probes=1))
    meshes = [capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP32), capi.GpuMesh(other, precision=capi.TLM_PRECISION_FP32)]
    b = capi.GpuBatch(meshes)
    b.set_variant(1)
    b.run(t["n_timesteps"])
    batched = (meshes[0].power_surfaces(), meshes[0].mode_outputs())
    b.close()
    for g in meshes:
        g.close()
    assert np.array_equal(batched[0], res[capi.TLM_PRECISION_FP32][0])
    assert np.array_equal(batched[1], res[capi.TLM_PRECISION_FP32][1])


@pytest.mark.gpu
def test_gpu_rejects_bad_arguments(gpu_lib):
    for key, value in (("ps_face_code", 9), ("mode_comp", 7), ("mode_face_out", 10 ** 6)):
        t = build_tables(spec_with_outputs(steps=10))
        t[key] = t[key].copy()
        t[key][0] = value
        with pytest.raises(capi.TLMError) as e:
            with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
                g.run(1)
        assert "TLM_E_BADARG" in str(e.value)
