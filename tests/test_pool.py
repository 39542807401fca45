"""The library's device-memory cache: buffers of destroyed meshes are reused
by later meshes, and a mesh built on reused (dirty) memory computes exactly
what one built on fresh memory does."""
import numpy as np
import pytest

from ggi_tlm_b200 import capi, cases
from ggi_tlm_b200.problem import build_tables

pytestmark = pytest.mark.gpu


def run(t, precision, steps):
    with capi.GpuMesh(t, precision=precision) as g:
        g.run(steps)
        return g.cell_output(), g.dft(), g.links()


def test_reused_memory_gives_identical_results(gpu_lib):
    capi.pool_release()
    assert capi.pool_cached_bytes() == 0
    a = build_tables(cases.pml_spheres(n=28, pml=4, n_spheres=3, steps=80, n_probes=4, n_freq=3, dft_size=8,
                                       rmin=2, rmax=4))
    b = build_tables(cases.debye_slabs(nx=26, ny=22, nz=40, pml=4, n_slabs=2, thickness=3, steps=80, n_freq=3,
                                       dft_size=8, margin=3))
    ref_a = run(a, capi.TLM_PRECISION_FP64, 80)
    cached = capi.pool_cached_bytes()
    assert cached > 0  # the destroyed mesh's buffers stay cached
    ref_b = run(b, capi.TLM_PRECISION_FP32, 80)  # runs on reused, dirty blocks
    again_a = run(a, capi.TLM_PRECISION_FP64, 80)
    for x, y in zip(ref_a, again_a):
        assert np.array_equal(x, y)
    capi.pool_release()
    fresh_b = run(b, capi.TLM_PRECISION_FP32, 80)  # fresh blocks from the driver
    for x, y in zip(ref_b, fresh_b):
        assert np.array_equal(x, y)
    capi.pool_release()
    assert capi.pool_cached_bytes() == 0
