"""Frequency output volumes (OUTPUT/frequency_output_volumes.F90:309-390):
the cells of a volume become output cells that keep no time series, and on
each output step (output.F90:564-598) value += field * exp(-j 2 pi f t) at
the time of the cell outputs.

CPU: the tables (numbering, series flags, CSR lists, cell spacing) and the
oracle restatement against a vectorised form of the same sum.  GPU: FP64
against the oracle at 1e-10, FP32 against FP64, batched against solo, the
probes unchanged next to the volumes, and argument errors."""
import os
import sys

import numpy as np
import pytest

from ggi_tlm_b200 import cases
from ggi_tlm_b200.problem import Block, FrequencyOutputVolume, build_tables, probe_series

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import oracle  # noqa: E402


def spec_with_volumes(steps=80):
    spec = cases.pml_spheres(n=24, pml=4, n_spheres=3, steps=steps, n_probes=4, n_freq=3, dft_size=6, rmin=2.0,
                             rmax=3.5)
    spec.frequency_output_volumes = [
        # free space, sphere and PML cells, every second cell, gated steps
        FrequencyOutputVolume(Block(2, 9, 3, 12, 4, 20), [1e9, 3e9], "Ez", first_step=5, last_step=70, interval=3,
                              every=2),
        # a line through both x PML slabs, every step
        FrequencyOutputVolume(Block(1, 24, 10, 10, 12, 12), [2e9], "Hx"),
    ]
    return spec


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_tables():
    spec = spec_with_volumes()
    t = build_tables(spec)
    n_pts = len([o for o in spec.outputs if o.face == "centre"])
    assert t["n_vdft"] == 3
    assert list(t["vdft_cell_ptr"]) == [0, 180, 360, 384]  # 4*5*9 cells twice, then 24
    assert int(t["out_keep"].sum()) == n_pts
    assert t["n_out_cells"] == 180 + 24 + n_pts
    out = t["vdft_cell_out"]
    assert out.min() >= 1 and out.max() <= t["n_out_cells"]
    assert np.all(np.diff(out[:180]) > 0)  # traversal order
    assert np.array_equal(out[:180], out[180:360])  # same cells for both frequencies
    assert not np.any(t["out_keep"][out - 1])  # volume cells keep no series
    assert list(t["vdft_first"]) == [5, 5, 1] and list(t["vdft_last"]) == [70, 70, 80]
    assert list(t["vdft_interval"]) == [3, 3, 1] and list(t["vdft_comp"]) == [3, 3, 4]
    with pytest.raises(ValueError):
        bad = spec_with_volumes()
        bad.frequency_output_volumes[0].component = "Jx"
        build_tables(bad)


def test_oracle_volume_dft_and_probes():
    spec = spec_with_volumes()
    t = build_tables(spec)
    hist = oracle.Oracle(t).run(t["n_timesteps"])
    v = oracle.volume_dft(t, hist)
    # the same sum, vectorised over the steps
    ptr, steps = t["vdft_cell_ptr"], np.arange(1, t["n_timesteps"] + 1)
    want = []
    for k in range(t["n_vdft"]):
        cells = t["vdft_cell_out"][ptr[k]:ptr[k + 1]] - 1
        on = (steps >= t["vdft_first"][k]) & (steps <= t["vdft_last"][k]) & (
            (steps - t["vdft_first"][k]) % t["vdft_interval"][k] == 0)
        ph = np.exp(-2j * np.pi * t["vdft_freq"][k] * (steps - 1) * t["dt"]) * on
        want.append(ph @ hist[:, cells, t["vdft_comp"][k] - 1])
    want = np.concatenate(want)
    assert np.abs(v).max() > 0
    assert rel(v, want) < 1e-12
    # volume outputs change no probe
    base = spec_with_volumes()
    base.frequency_output_volumes = []
    tb = build_tables(base)
    assert np.array_equal(probe_series(tb, oracle.Oracle(tb).run(tb["n_timesteps"])), probe_series(t, hist))


@pytest.mark.gpu
def test_gpu_fp64_matches_oracle(gpu_lib):
    from ggi_tlm_b200 import capi

    t = build_tables(spec_with_volumes())
    hist = oracle.Oracle(t).run(t["n_timesteps"])
    want = oracle.volume_dft(t, hist)
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.run(t["n_timesteps"])
        got = g.volume_dft()
        co = g.cell_output()
    assert co.shape[1] == int(t["out_keep"].sum())  # only the probes keep a series
    ptr = t["vdft_cell_ptr"]
    for k in range(t["n_vdft"]):
        assert rel(got[ptr[k]:ptr[k + 1]], want[ptr[k]:ptr[k + 1]]) < 1e-10
    ps, po = probe_series(t, co), probe_series(t, hist)
    for a, b in zip(ps, po):
        assert rel(a, b) < 1e-10


@pytest.mark.gpu
def test_gpu_fp32_close_to_fp64_and_batch_equals_solo(gpu_lib):
    from ggi_tlm_b200 import capi

    t = build_tables(spec_with_volumes(steps=120))
    res = {}
    for prec in (capi.TLM_PRECISION_FP32, capi.TLM_PRECISION_FP64):
        with capi.GpuMesh(t, precision=prec) as g:
            g.set_variant(1)
            g.run(t["n_timesteps"])
            res[prec] = g.volume_dft()
    assert rel(res[capi.TLM_PRECISION_FP32], res[capi.TLM_PRECISION_FP64]) < 1e-3
    # the same mesh in a batch with another mesh: bit-identical to solo
    other = build_tables(cases.pml_point_source(20, steps=60, pml=3, n_probes=1))
    meshes = [capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP32), capi.GpuMesh(other, precision=capi.TLM_PRECISION_FP32)]
    b = capi.GpuBatch(meshes)
    b.set_variant(1)
    b.run(t["n_timesteps"])
    batched = meshes[0].volume_dft()
    b.close()
    for g in meshes:
        g.close()
    assert np.array_equal(batched, res[capi.TLM_PRECISION_FP32])


@pytest.mark.gpu
def test_gpu_rejects_bad_volume_arguments(gpu_lib):
    from ggi_tlm_b200 import capi

    for key, value in (("vdft_comp", 7), ("vdft_interval", 0), ("vdft_cell_out", 10 ** 6)):
        t = build_tables(spec_with_volumes(steps=10))
        t[key] = t[key].copy()
        t[key][0] = value
        with pytest.raises(capi.TLMError) as e:
            with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
                g.run(1)
        assert "TLM_E_BADARG" in str(e.value)
