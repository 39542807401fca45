"""Batched execution: uneven meshes advanced by one launch per kernel type
per step give exactly the results of running each mesh on its own."""
import numpy as np
import pytest

from ggi_tlm_b200 import capi, cases
from ggi_tlm_b200.problem import build_tables, probe_series

import oracle as O

pytestmark = pytest.mark.gpu


def uneven_tables(n=5, seed=3):
    specs = cases.batch_boxes(n_boxes=n, edge=(18, 33), steps=(40, 90), pml=3, max_spheres=3, seed=seed)
    specs[0].huygens = None
    return [build_tables(s) for s in specs]


@pytest.mark.parametrize("precision", [capi.TLM_PRECISION_FP32, capi.TLM_PRECISION_FP64])
def test_batch_equals_individual_runs(gpu_lib, precision):
    tabs = uneven_tables()
    solo = []
    for t in tabs:
        with capi.GpuMesh(t, precision=precision) as g:
            g.set_variant(1)
            g.run(t["n_timesteps"])
            solo.append((g.cell_output(), g.links()))
    meshes = [capi.GpuMesh(t, precision=precision) for t in tabs]
    with capi.GpuBatch(meshes) as b:
        b.set_variant(1)
        b.run(17)  # partial, then the rest (meshes finish at different steps)
        b.run(1000)
        ms, cu, launches = b.last_run()
        assert cu == sum(t["nx"] * t["ny"] * t["nz"] * (t["n_timesteps"] - 17) for t in tabs)
        assert launches > 0
    for g, t, (co, li) in zip(meshes, tabs, solo):
        assert g.step == t["n_timesteps"]
        assert np.array_equal(g.cell_output(), co)
        assert np.array_equal(g.links(), li)
        g.close()
    if precision == capi.TLM_PRECISION_FP64:
        t = tabs[1]
        o = O.Oracle(t)
        po = probe_series(t, o.run(t["n_timesteps"]))
        pg = probe_series(t, solo[1][0])
        for i in range(len(po)):
            assert np.linalg.norm(pg[i] - po[i]) <= 1e-10 * max(np.linalg.norm(po[i]), 1e-300)


def test_batch_rejects_mixed_precision(gpu_lib):
    tabs = uneven_tables(2)
    a = capi.GpuMesh(tabs[0], precision=capi.TLM_PRECISION_FP32)
    b = capi.GpuMesh(tabs[1], precision=capi.TLM_PRECISION_FP64)
    with pytest.raises(capi.TLMError):
        capi.GpuBatch([a, b])
    a.close()
    b.close()


@pytest.mark.parametrize("precision", [capi.TLM_PRECISION_FP32, capi.TLM_PRECISION_FP64])
def test_batch_members_change_between_runs(gpu_lib, precision):
    """Meshes leave and join a running batch (tlm_gpu_batch_set_members):
    every mesh still gives its solo results bit for bit, a leaver can run on
    its own, and the batch keeps working across the changes."""
    tabs = uneven_tables(n=5, seed=4)
    solo = []
    for t in tabs:
        with capi.GpuMesh(t, precision=precision) as g:
            g.set_variant(1)
            g.run(t["n_timesteps"])
            solo.append(g.cell_output())
    m = [capi.GpuMesh(t, precision=precision) for t in tabs]
    for g in m:
        g.set_variant(1)
    with capi.GpuBatch(m[:3]) as b:
        b.set_variant(1)
        b.run(11)
        b.set_members([m[1], m[2], m[3]])  # m0 leaves, m3 joins
        m[0].run(5)  # the leaver runs alone
        b.run(13)
        b.set_members([m[0], m[2], m[3], m[4]])  # m0 back, m1 leaves, m4 joins
        b.run(1000)
        m[1].run(tabs[1]["n_timesteps"] - m[1].step)
        b.synchronize()
    for g, t, co in zip(m, tabs, solo):
        assert g.step == t["n_timesteps"]
        assert np.array_equal(g.cell_output(), co)
    for g in m:
        g.close()
