"""PML cells inside a non-dispersive volume material
(TLM_SOLVER/scatter_PML_material.F90:22-534).

No golden series of the reference covers this update, so the oracle's
restatement is checked physically first: a lossy dielectric substrate that
runs into the PML must look, from inside the box, like the same substrate in
an unbounded domain (a box so large that its boundary is not seen within the
run).  Cutting the substrate at the PML instead leaves a reflecting
discontinuity, which the same comparison sees.  The GPU path is then checked
against the oracle.
"""
import numpy as np
import pytest

from ggi_tlm_b200 import capi, cases
from ggi_tlm_b200.problem import (Block, ExcitationFunction, Sfilter, UnsupportedFeature, VolumeMaterial, build_tables,
                                  probe_series)

import oracle as O

N, PML, TOP, STEPS = 28, 6, 10, 160


def oracle_probes(t, steps=None):
    return probe_series(t, O.Oracle(t).run(t["n_timesteps"] if steps is None else steps))


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def unbounded():
    t = build_tables(cases.pml_dielectric_slab(N, PML, STEPS, slab_top=TOP, pad=40))
    assert t["n_pml_material_cells"] == 0
    return oracle_probes(t)


def test_oracle_pml_in_dielectric_absorbs(unbounded):
    t = build_tables(cases.pml_dielectric_slab(N, PML, STEPS, slab_top=TOP))
    assert t["n_pml_material_cells"] > 0
    p = oracle_probes(t)
    err = [rel(p[i], unbounded[i]) for i in range(3)]
    assert max(err) < 0.02, err  # measured: 8.5e-3, 1.4e-3, 1.7e-3
    # the substrate cut at the PML reflects: much further from the unbounded answer
    spec = cases.pml_dielectric_slab(N, PML, STEPS, slab_top=TOP)
    spec.material_regions = [(1, Block(PML + 1, N - PML, PML + 1, N - PML, PML + 1, TOP))]
    tc = build_tables(spec)
    assert tc["n_pml_material_cells"] == 0
    pc = oracle_probes(tc)
    assert rel(pc[0], unbounded[0]) > 10 * err[0]


def test_oracle_pml_material_in_vacuum_equals_free_space_pml():
    """With eps_r = mu_r = 1 and no loss the stubs vanish and the
    second-order recursions must reproduce the free-space PML update
    (scatter_PML.F90, pinned by the TEM_PML_TEST golden series)."""
    s1 = cases.pml_dielectric_slab(N, PML, 1500, eps_r=1.0, sigma=0.0, slab_top=TOP)
    s0 = cases.pml_dielectric_slab(N, PML, 1500, eps_r=1.0, sigma=0.0, slab_top=TOP)
    s0.materials, s0.material_regions = [], []
    t1, t0 = build_tables(s1), build_tables(s0)
    assert t1["n_pml_material_cells"] > 0 and t0["n_pml_material_cells"] == 0
    o1, o0 = O.Oracle(t1), O.Oracle(t0)
    p1, p0 = probe_series(t1, o1.run(1500)), probe_series(t0, o0.run(1500))
    assert max(rel(p1[i], p0[i]) for i in range(3)) < 1e-9  # measured 9.5e-11
    l1, l0 = o1.links(), o0.links()
    assert np.abs(l1 - l0).max() < 1e-10 * np.abs(l0).max()


def test_oracle_pml_in_dielectric_decays():
    """A source without DC content (differential Gaussian) leaves nothing
    behind: after 3000 steps the fields have left through the PML."""
    spec = cases.pml_dielectric_slab(N, PML, 3000, slab_top=TOP)
    spec.functions = [ExcitationFunction("differential_gaussian", (1.0, 0.05e-9, 0.2e-9))]
    t = build_tables(spec)
    p = oracle_probes(t)
    assert np.all(np.isfinite(p))
    assert np.abs(p[:, -500:]).max() < 1e-3 * np.abs(p).max()


def test_tables_reject_what_the_reference_stops_on():
    spec = cases.pml_dielectric_slab(N, PML, 10, slab_top=TOP)
    spec.materials = [VolumeMaterial.debye(3.0, [10.0], [1e-10])]
    with pytest.raises(UnsupportedFeature, match="dispersive"):
        build_tables(spec)
    spec.materials = [VolumeMaterial(1, Sfilter(1.0, [1.0], [1.0]), 0.0, Sfilter(1.0, [1.0], [1.0]), 0.0)]
    with pytest.raises(UnsupportedFeature, match="PEC/PMC"):
        build_tables(spec)


def _gpu(t, precision, steps, chunks=(60,)):
    with capi.GpuMesh(t, precision=precision) as g:
        done = 0
        for c in chunks:
            g.run(c)
            done += c
        g.run(steps - done)
        return probe_series(t, g.cell_output()), g.links()


@pytest.mark.gpu
def test_gpu_pml_material_matches_oracle(gpu_lib):
    t = build_tables(cases.pml_dielectric_slab(N, PML, 400, slab_top=TOP))
    o = O.Oracle(t)
    po = probe_series(t, o.run(400))
    lo = o.links()
    pg, lg = _gpu(t, capi.TLM_PRECISION_FP64, 400)
    assert max(rel(pg[i], po[i]) for i in range(3)) < 1e-10
    assert np.max(np.abs(lg - lo)) <= 1e-10 * np.max(np.abs(lo))
    p32, _ = _gpu(t, capi.TLM_PRECISION_FP32, 400)
    assert max(rel(p32[i], pg[i]) for i in range(3)) < 1e-4


@pytest.mark.gpu
def test_gpu_pml_material_in_a_batch_equals_solo(gpu_lib):
    tabs = [build_tables(cases.pml_dielectric_slab(N, PML, 120, slab_top=TOP)),
            build_tables(cases.pml_spheres(n=20, pml=4, n_spheres=2, steps=90, n_probes=3, n_freq=2, dft_size=6,
                                           rmin=2, rmax=3)),
            build_tables(cases.pml_dielectric_slab(32, 5, 100, eps_r=2.5, sigma=0.0, slab_top=12))]
    for prec in (capi.TLM_PRECISION_FP64, capi.TLM_PRECISION_FP32):
        solo = []
        for t in tabs:
            with capi.GpuMesh(t, precision=prec) as g:
                g.set_variant(1)
                g.run(t["n_timesteps"])
                solo.append(g.cell_output())
        meshes = [capi.GpuMesh(t, precision=prec) for t in tabs]
        with capi.GpuBatch(meshes) as b:
            b.set_variant(1)
            b.run(1000)
        for g, co in zip(meshes, solo):
            assert np.array_equal(g.cell_output(), co)
            g.close()


@pytest.mark.gpu
def test_gpu_pml_material_needs_sigma(gpu_lib):
    t = dict(build_tables(cases.pml_dielectric_slab(N, PML, 10, slab_top=TOP)))
    t["n_pml_material_cells"] = 0  # the binding then skips tlm_gpu_set_pml_sigma
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        with pytest.raises(capi.TLMError) as e:
            g.run(1)
        assert e.value.code == capi.TLM_E_BADARG and "set_pml_sigma" in str(e.value)
