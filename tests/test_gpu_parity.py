"""GPU path (through the C-ABI) against the CPU oracle and the reference's
golden series.

Tolerances: plain FP64 GPU vs oracle <= 1e-10 relative L2 per probe series
(the FP64 path differs from the reference's arithmetic only by FMA
contraction and by the pull-form connect, which forwards the neighbour's
pulse instead of computing (a+b)-a); FP32 vs FP64 GPU <= 1e-4.
"""
import os

import numpy as np
import pytest

from ggi_tlm_b200 import capi, cases
from ggi_tlm_b200.problem import build_tables, probe_series

import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FP64_TOL = 1e-10
FP32_TOL = 1e-4


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / nb if nb > 0 else np.linalg.norm(a - b)


def per_probe(a, b):
    return max(rel_l2(a[i], b[i]) for i in range(a.shape[0]))


def run_gpu(t, precision, steps=None, chunks=None):
    steps = t["n_timesteps"] if steps is None else steps
    with capi.GpuMesh(t, precision=precision) as g:
        for n in (chunks or [steps]):
            g.run(n)
        co = g.cell_output()
        dft = g.dft()
        links = g.links()
    return probe_series(t, co), dft, links


def run_oracle(t, steps=None):
    steps = t["n_timesteps"] if steps is None else steps
    o = O.Oracle(t)
    co = o.run(steps)
    return probe_series(t, co), o.dft(), o.links()


@pytest.mark.parametrize("name", sorted(cases.KAT_CASES))
def test_gpu_fp64_known_answer(gpu_lib, name):
    t = build_tables(cases.KAT_CASES[name]())
    pg, _, lg = run_gpu(t, capi.TLM_PRECISION_FP64)
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    v = np.where(np.abs(pg[0]) < 1e-30, 0.0, pg[0])
    assert rel_l2(v, d["value"]) < 5e-7
    if t["nx"] * t["ny"] * t["nz"] * t["n_timesteps"] < 5e7:  # the oracle finishes in seconds
        po, _, lo = run_oracle(t)
        assert per_probe(pg, po) < FP64_TOL
        assert np.max(np.abs(lg - lo)) <= 1e-10 * max(np.max(np.abs(lo)), 1e-300)


def _check_case(t, steps=None):
    pg, dg, lg = run_gpu(t, capi.TLM_PRECISION_FP64, steps)
    po, do, lo = run_oracle(t, steps)
    assert per_probe(pg, po) < FP64_TOL
    if do.size:
        assert rel_l2(dg, do) < FP64_TOL
    scale = max(np.max(np.abs(lo)), 1e-300)
    assert np.max(np.abs(lg - lo)) <= 1e-10 * scale
    return pg, po


def test_gpu_fp64_pec_box(gpu_lib):
    t = build_tables(cases.pec_box(n=16, steps=240))
    _check_case(t)


def test_gpu_fp64_pec_box_config_size(gpu_lib):
    """The parity configuration itself: 40^3 PEC box, 2000 steps, 12 probes."""
    t = build_tables(cases.pec_box())
    _check_case(t)


def test_gpu_fp64_pml_spheres_huygens_dft(gpu_lib):
    spec = cases.pml_spheres(n=28, pml=5, n_spheres=4, steps=260, n_probes=6, n_freq=5, dft_size=8, rmin=2.0,
                             rmax=4.0)
    t = build_tables(spec)
    assert t["n_pml_cells"] > 0 and t["n_materials"] > 0 and t["hs_n"] > 0 and t["n_dft"] == 5
    _check_case(t)


def test_gpu_fp64_debye_slabs(gpu_lib):
    spec = cases.debye_slabs(nx=26, ny=22, nz=40, pml=4, n_slabs=2, thickness=3, steps=300, n_freq=3,
                             dft_size=6, margin=2)
    t = build_tables(spec)
    assert t["mat_eps_order"].max() == 3  # 2-pole Debye -> order-3 Z filters
    _check_case(t)


@pytest.mark.parametrize("dims", [(27, 22, 19), (5, 33, 9), (1, 1, 64), (33, 1, 7)])
def test_gpu_fp64_ragged_boxes(gpu_lib, dims):
    nx, ny, nz = dims
    pml = 2 if min(dims) > 8 else 0
    spec = cases.pml_point_source(nx, ny, nz, pml=pml, steps=90, n_spheres=2 if min(dims) > 12 else 0, seed=11,
                                  n_probes=3)
    spec.R = (-1.0, 0.5, 1.0, -0.3, 0.0, -1.0)
    _check_case(build_tables(spec))


def test_gpu_fp32_vs_fp64(gpu_lib):
    spec = cases.pml_spheres(n=32, pml=6, n_spheres=3, steps=400, n_probes=8, n_freq=4, dft_size=8, rmin=2.0,
                             rmax=4.0)
    t = build_tables(spec)
    p64, d64, _ = run_gpu(t, capi.TLM_PRECISION_FP64)
    p32, d32, _ = run_gpu(t, capi.TLM_PRECISION_FP32)
    assert per_probe(p32, p64) < FP32_TOL
    assert rel_l2(d32, d64) < FP32_TOL


def test_gpu_fp32_vs_fp64_debye(gpu_lib):
    spec = cases.debye_slabs(nx=24, ny=24, nz=48, pml=4, n_slabs=2, thickness=3, steps=500, n_freq=2,
                             dft_size=6, margin=2)
    t = build_tables(spec)
    p64, _, _ = run_gpu(t, capi.TLM_PRECISION_FP64)
    p32, _, _ = run_gpu(t, capi.TLM_PRECISION_FP32)
    assert per_probe(p32, p64) < FP32_TOL


def test_gpu_run_split_and_graph_paths_identical(gpu_lib):
    """Graph replay (bundles of steps), ragged remainders and the per-step
    timing path produce bit-identical results."""
    t = build_tables(cases.pml_spheres(n=20, pml=3, n_spheres=2, steps=70, n_probes=3, n_freq=2, dft_size=4,
                                       rmin=2.0, rmax=3.0))
    a, da, la = run_gpu(t, capi.TLM_PRECISION_FP64, chunks=[70])
    b, db, lb = run_gpu(t, capi.TLM_PRECISION_FP64, chunks=[3, 17, 8, 42])
    assert np.array_equal(a, b) and np.array_equal(da, db) and np.array_equal(la, lb)
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.set_timing(True)
        g.run(70)
        total, cell = g.last_run_time()
        assert total > 0 and cell > 0
        c = probe_series(t, g.cell_output())
    assert np.array_equal(a, c)


def test_gpu_rejects_unsupported_and_bad_calls(gpu_lib):
    t = build_tables(cases.pec_box(n=8, steps=10))
    with capi.GpuMesh(t) as g:
        with pytest.raises(capi.TLMError) as e:
            capi._check(capi._lib.tlm_gpu_run(g.h, 2, 1))  # steps must start at 1
        assert e.value.code == -5
        with pytest.raises(capi.TLMError):
            g.run(11)  # beyond n_timesteps
    # a PML cell inside a PEC volume material is rejected up front (scatter.F90:559-567)
    bad = dict(t)
    bad["sp_pml"] = np.array(t["sp_pml"]).copy()
    bad["n_pml_params"] = 1
    bad["pml_params"] = np.ones((1, 15))
    bad["n_pml_cells"] = 1
    bad["pml_cell_param"] = np.array([1], np.int32)
    bad["n_materials"] = 1
    for k in ("mat_type",):
        bad[k] = np.array([1], np.int32)
    bad["sp_material"] = np.ones_like(np.array(t["sp_material"]))
    bad["sp_pml"][0] = 1
    with pytest.raises(capi.TLMError) as e:
        with capi.GpuMesh(bad) as g:
            g.run(1)
    assert e.value.code == -2


@pytest.mark.parametrize("precision", [capi.TLM_PRECISION_FP32, capi.TLM_PRECISION_FP64])
def test_gpu_bulk_variants_bit_identical(gpu_lib, precision):
    """Every bulk-kernel configuration (register-pipelined and TMA-staged with
    different tiles / ring depths) computes bit-identical results, on a mesh
    whose plane interiors are not multiples of any tile size."""
    t = build_tables(cases.pml_spheres(n=37, pml=4, n_spheres=3, steps=50, n_probes=5, n_freq=2, dft_size=6,
                                       rmin=2.0, rmax=4.0))
    ref = None
    for v in range(capi.num_variants()):
        with capi.GpuMesh(t, precision=precision) as g:
            g.set_variant(v)
            g.run(50)
            res = (g.cell_output(), g.dft(), g.links())
        if ref is None:
            ref = res
        else:
            for a, b in zip(ref, res):
                assert np.array_equal(a, b), f"variant {v} differs"
    if precision == capi.TLM_PRECISION_FP64:
        po, do, lo = run_oracle(t, 50)
        assert per_probe(probe_series(t, ref[0]), po) < FP64_TOL
