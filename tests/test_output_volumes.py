"""Time-domain output volumes: each cell's field (OUTPUT/output_volumes.F90),
the volume average (output_volume_averages.F90) and the volume peak
(output_volume_peak.F90) on gated output steps, from the current-step
cell output rows.

CPU: the tables and the oracle restatement against numpy forms of the same
reductions.  GPU: FP64 against the oracle, FP32 against FP64, batched
against solo, and argument errors."""
import os
import sys

import numpy as np
import pytest

from ggi_tlm_b200 import capi, cases
from ggi_tlm_b200.problem import Block, OutputVolume, build_tables, probe_series

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import oracle  # noqa: E402


def spec_with_volumes(steps=80):
    spec = cases.pml_spheres(n=24, pml=4, n_spheres=3, steps=steps, n_probes=4, n_freq=3, dft_size=6, rmin=2.0,
                             rmax=3.5)
    blk = Block(2, 12, 3, 14, 6, 18)  # free space, sphere and PML cells
    spec.output_volumes = [
        OutputVolume(blk, "Ey", "field", first_step=4, interval=5, every=2),
        OutputVolume(blk, "Ey", "average"),
        OutputVolume(blk, "Hx", "peak", last_step=60, interval=2),
        OutputVolume(Block(1, 24, 12, 12, 12, 12), "Ex", "average", first_step=10),  # a line through the PML
    ]
    return spec


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_tables():
    spec = spec_with_volumes()
    t = build_tables(spec)
    assert t["n_ovol"] == 4 and list(t["ovol_kind"]) == [0, 1, 2, 1]
    ptr = t["ovol_cell_ptr"]
    assert ptr[1] - ptr[0] == 6 * 6 * 7 and ptr[2] - ptr[1] == 11 * 12 * 13 and ptr[4] - ptr[3] == 24
    n_pts = len([o for o in spec.outputs if o.face == "centre"])
    assert int(t["out_keep"].sum()) == n_pts  # volume cells keep no time series
    with pytest.raises(ValueError):
        bad = spec_with_volumes()
        bad.output_volumes[0].kind = "rms"
        build_tables(bad)


def test_oracle_reductions():
    t = build_tables(spec_with_volumes())
    hist = oracle.Oracle(t).run(t["n_timesteps"])
    r = oracle.output_volumes(t, hist)
    ptr = t["ovol_cell_ptr"]
    cells = [t["ovol_cell_out"][ptr[k]:ptr[k + 1]] - 1 for k in range(4)]
    assert r[0].shape == (16, 6 * 6 * 7)  # steps 4, 9, ..., 79
    assert np.array_equal(r[0], hist[3::5, cells[0], 1])
    want_avg = hist[:, cells[1], 1].mean(axis=1)
    want_avg[np.abs(want_avg) < 1e-30] = 0.0
    assert np.allclose(r[1], want_avg, rtol=1e-12, atol=0)
    assert np.array_equal(r[2], np.abs(hist[0:60:2, cells[2], 3]).max(axis=1))
    assert r[3].shape == (71,) and np.abs(r[1]).max() > 0 and np.abs(r[2]).max() > 0


@pytest.mark.gpu
def test_gpu_fp64_matches_oracle(gpu_lib):
    t = build_tables(spec_with_volumes())
    hist = oracle.Oracle(t).run(t["n_timesteps"])
    want = oracle.output_volumes(t, hist)
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.run(t["n_timesteps"])
        got = g.output_volumes()
        ps = probe_series(t, g.cell_output())
    for k, (a, b) in enumerate(zip(got, want)):
        assert a.shape == b.shape
        assert rel(a, b) < 1e-10, k
    for a, b in zip(ps, probe_series(t, hist)):
        assert rel(a, b) < 1e-10


@pytest.mark.gpu
def test_gpu_fp32_and_batch_equals_solo(gpu_lib):
    t = build_tables(spec_with_volumes(steps=100))
    res = {}
    for prec in (capi.TLM_PRECISION_FP32, capi.TLM_PRECISION_FP64):
        with capi.GpuMesh(t, precision=prec) as g:
            g.set_variant(1)
            g.run(t["n_timesteps"])
            res[prec] = g.output_volumes()
    for k in range(3):
        assert rel(res[capi.TLM_PRECISION_FP32][k], res[capi.TLM_PRECISION_FP64][k]) < 1e-3, k
    other = build_tables(cases.pml_point_source(20, steps=40, pml=3, n_probes=1))
    meshes = [capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP32), capi.GpuMesh(other, precision=capi.TLM_PRECISION_FP32)]
    b = capi.GpuBatch(meshes)
    b.set_variant(1)
    b.run(t["n_timesteps"])
    batched = meshes[0].output_volumes()
    b.close()
    for g in meshes:
        g.close()
    for a, c in zip(batched, res[capi.TLM_PRECISION_FP32]):
        assert np.array_equal(a, c)


@pytest.mark.gpu
def test_gpu_rejects_bad_volume_arguments(gpu_lib):
    for key, value in (("ovol_kind", 3), ("ovol_comp", 7), ("ovol_interval", 0), ("ovol_cell_out", 10 ** 6)):
        t = build_tables(spec_with_volumes(steps=10))
        t[key] = t[key].copy()
        t[key][0] = value
        with pytest.raises(capi.TLMError) as e:
            with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
                g.run(1)
        assert "TLM_E_BADARG" in str(e.value)
