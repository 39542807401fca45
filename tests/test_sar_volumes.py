"""SAR volumes (OUTPUT/SAR_volumes.F90:257-330): every step each cell of the
volume accumulates the DFT of Ex, Ey, Ez times dt at the cell-output time;
write_SAR_volumes turns them into SAR on the host.

CPU: the tables and the oracle restatement against a vectorised form.  GPU:
FP64 against the oracle, FP32 against FP64, batched against solo, and an
argument error."""
import os
import sys

import numpy as np
import pytest

from ggi_tlm_b200 import capi, cases
from ggi_tlm_b200.problem import Block, SARVolume, build_tables

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import oracle  # noqa: E402


def spec_with_sar(steps=80):
    spec = cases.pml_spheres(n=24, pml=4, n_spheres=3, steps=steps, n_probes=4, n_freq=3, dft_size=6, rmin=2.0,
                             rmax=3.5)
    spec.sar_volumes = [SARVolume(Block(3, 14, 4, 15, 6, 18), [1.5e9, 4e9], every=2),  # sphere, free and PML cells
                        SARVolume(Block(10, 12, 10, 12, 10, 12), [2e9])]
    return spec


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_tables_and_oracle():
    t = build_tables(spec_with_sar())
    ptr = t["sar_cell_ptr"]
    assert t["n_sar"] == 3 and list(ptr) == [0, 252, 504, 531]  # 6*6*7 twice, then 27
    assert not np.any(t["out_keep"][t["sar_cell_out"] - 1])
    hist = oracle.Oracle(t).run(t["n_timesteps"])
    got = oracle.sar_volumes(t, hist)
    steps = np.arange(t["n_timesteps"])
    want = []
    for k in range(t["n_sar"]):
        cells = t["sar_cell_out"][ptr[k]:ptr[k + 1]] - 1
        ph = np.exp(-2j * np.pi * t["sar_freq"][k] * steps * t["dt"]) * t["dt"]
        want.append(np.einsum("s,scx->cx", ph, hist[:, cells, 0:3]))
    want = np.concatenate(want)
    assert np.abs(got).max() > 0
    assert rel(got, want) < 1e-12


@pytest.mark.gpu
def test_gpu_fp64_matches_oracle(gpu_lib):
    t = build_tables(spec_with_sar())
    want = oracle.sar_volumes(t, oracle.Oracle(t).run(t["n_timesteps"]))
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.run(t["n_timesteps"])
        got = g.sar_volumes()
    ptr = t["sar_cell_ptr"]
    for k in range(t["n_sar"]):
        assert rel(got[ptr[k]:ptr[k + 1]], want[ptr[k]:ptr[k + 1]]) < 1e-10, k


@pytest.mark.gpu
def test_gpu_fp32_and_batch_equals_solo(gpu_lib):
    t = build_tables(spec_with_sar(steps=100))
    res = {}
    for prec in (capi.TLM_PRECISION_FP32, capi.TLM_PRECISION_FP64):
        with capi.GpuMesh(t, precision=prec) as g:
            g.set_variant(1)
            g.run(t["n_timesteps"])
            res[prec] = g.sar_volumes()
    assert rel(res[capi.TLM_PRECISION_FP32], res[capi.TLM_PRECISION_FP64]) < 1e-3
    other = build_tables(cases.pml_point_source(20, steps=40, pml=3, n_probes=1))
    meshes = [capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP32), capi.GpuMesh(other, precision=capi.TLM_PRECISION_FP32)]
    b = capi.GpuBatch(meshes)
    b.set_variant(1)
    b.run(t["n_timesteps"])
    batched = meshes[0].sar_volumes()
    b.close()
    for g in meshes:
        g.close()
    assert np.array_equal(batched, res[capi.TLM_PRECISION_FP32])


@pytest.mark.gpu
def test_gpu_rejects_bad_sar_cell(gpu_lib):
    t = build_tables(spec_with_sar(steps=10))
    t["sar_cell_out"] = t["sar_cell_out"].copy()
    t["sar_cell_out"][0] = 10 ** 6
    with pytest.raises(capi.TLMError) as e:
        with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
            g.run(1)
    assert "TLM_E_BADARG" in str(e.value)
