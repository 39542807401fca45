"""set_small_to_zero (TLM_SOLVER/TLM_set_small_to_zero.F90:34-68, called at
run_TLM.F90:236-238): every n steps, incident pulses with |V| < value become
0 before the excitation.  The oracle is checked for its defining
properties on the CPU; the GPU path (solo and batched) against the oracle.
"""
import numpy as np
import pytest

from ggi_tlm_b200 import capi, cases
from ggi_tlm_b200.problem import build_tables, probe_series

import oracle as O

STEPS = 300
THRESHOLD = 1e-6  # changes the probe series of this case by ~1e-3 (checked below)


def spec(small=None):
    s = cases.pml_spheres(n=24, pml=4, n_spheres=2, steps=STEPS, n_probes=4, n_freq=3, dft_size=8, rmin=2, rmax=4)
    s.small_to_zero = small
    return s


def oracle_run(t):
    o = O.Oracle(t)
    return probe_series(t, o.run(t["n_timesteps"])), o.dft(), o.links()


def rel(a, b):
    return max(np.linalg.norm(a[i] - b[i]) / np.linalg.norm(b[i]) for i in range(len(b)))


def test_oracle_flush_properties():
    p0, d0, l0 = oracle_run(build_tables(spec()))
    # a zero threshold and a period longer than the run change nothing
    for small in ((1, 0.0), (STEPS + 1, 1.0)):
        p, d, li = oracle_run(build_tables(spec(small)))
        assert np.array_equal(p, p0) and np.array_equal(d, d0) and np.array_equal(li, l0)
    # a threshold below the signal changes the answer, but only a little
    p, _, _ = oracle_run(build_tables(spec((3, THRESHOLD))))
    assert 1e-5 < rel(p, p0) < 1e-2


def test_tables_reject_negative_flush_arguments():
    with pytest.raises(ValueError):
        build_tables(spec((-1, 1e-6)))
    with pytest.raises(ValueError):
        build_tables(spec((3, -1e-6)))


@pytest.mark.gpu
def test_gpu_flush_matches_oracle(gpu_lib):
    t = build_tables(spec((3, THRESHOLD)))
    po, do, lo = oracle_run(t)
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.run(100)
        g.run(STEPS - 100)  # graph replay across the split
        pg = probe_series(t, g.cell_output())
        dg, lg = g.dft(), g.links()
    assert rel(pg, po) < 1e-10
    assert np.linalg.norm(dg - do) <= 1e-10 * np.linalg.norm(do)
    assert np.max(np.abs(lg - lo)) <= 1e-10 * np.max(np.abs(lo))
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP32) as g:
        g.run(STEPS)
        p32 = probe_series(t, g.cell_output())
    assert rel(p32, po) < 1e-3


@pytest.mark.gpu
def test_gpu_flush_in_a_batch_equals_solo(gpu_lib):
    tabs = [build_tables(spec((3, THRESHOLD))), build_tables(spec()), build_tables(spec((5, 1e-5)))]
    solo = []
    for t in tabs:
        with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
            g.set_variant(1)
            g.run(STEPS)
            solo.append(g.cell_output())
    meshes = [capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) for t in tabs]
    with capi.GpuBatch(meshes) as b:
        b.set_variant(1)
        b.run(STEPS)
    for g, co in zip(meshes, solo):
        assert np.array_equal(g.cell_output(), co)
        g.close()


@pytest.mark.gpu
def test_gpu_flush_argument_errors(gpu_lib):
    t = build_tables(spec())
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        lib = capi._lib
        assert lib.tlm_gpu_set_small_to_zero(g.h, -1, 1e-6) == capi.TLM_E_BADARG
        assert lib.tlm_gpu_set_small_to_zero(g.h, 3, -1.0) == capi.TLM_E_BADARG
        assert lib.tlm_gpu_set_small_to_zero(g.h, 3, float("nan")) == capi.TLM_E_BADARG
        g.run(1)
        assert lib.tlm_gpu_set_small_to_zero(g.h, 3, 1e-6) == capi.TLM_E_STATE
