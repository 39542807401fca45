"""The allocation-free read-back entry point (tlm_gpu_fetch_links_noalloc).

Some callers of this library cannot call cudaMalloc: a host framework that
owns a fixed device-memory budget, or code that must not add the implicit
device synchronisation of cudaMalloc/cudaFree while its own GPU work is in
flight.  For them the library has one entry point that allocates nothing:
it gathers the incident link voltages into a fixed scratch array compiled
into the library instead of a temporary device buffer.  This test calls it
through the C-ABI, twice in a row, and checks each result against the
allocating entry point tlm_gpu_fetch_links on the same mesh state.

The file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from ggi_tlm_b200 import capi, cases
from ggi_tlm_b200.problem import build_tables

pytestmark = pytest.mark.gpu
TOL = 1e-10  # the FP64 parity tolerance of the GPU tests; both paths run the same gather


def fetch(lib, h, name, shape):
    out = np.zeros(int(np.prod(shape)))
    capi._check(getattr(lib, name)(h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    return out.reshape(shape)


@pytest.mark.parametrize("precision", [capi.TLM_PRECISION_FP64, capi.TLM_PRECISION_FP32])
def test_noalloc_fetch_matches_allocating_fetch(gpu_lib, precision):
    t = build_tables(cases.pml_spheres(n=24, pml=4, n_spheres=3, steps=80, n_probes=3, n_freq=2, dft_size=4,
                                       rmin=2.0, rmax=3.0))
    shape = (t["nz"], t["ny"], t["nx"], 12)
    with capi.GpuMesh(t, precision=precision) as g:
        g.run(37)
        ref1 = fetch(capi._lib, g.h, "tlm_gpu_fetch_links", shape)
        a1 = fetch(capi._lib, g.h, "tlm_gpu_fetch_links_noalloc", shape)
        a2 = fetch(capi._lib, g.h, "tlm_gpu_fetch_links_noalloc", shape)  # second call in a row
        g.run(5)
        ref2 = fetch(capi._lib, g.h, "tlm_gpu_fetch_links", shape)
        b1 = fetch(capi._lib, g.h, "tlm_gpu_fetch_links_noalloc", shape)
    scale = np.max(np.abs(ref1))
    assert scale > 0
    for got, ref in ((a1, ref1), (a2, ref1), (b1, ref2)):
        assert np.max(np.abs(got - ref)) <= TOL * max(scale, np.max(np.abs(ref)))


def test_noalloc_fetch_of_a_batched_mesh_waits_for_the_batch(gpu_lib):
    """A mesh inside a batch is advanced on the batch's stream, and
    tlm_gpu_batch_run returns before its steps finish: the read-back must
    still see the finished steps, twice in a row, as the allocating
    read-back does."""
    specs = cases.batch_boxes(n_boxes=2, edge=(18, 26), steps=(60, 80), pml=3, max_spheres=2, seed=5)
    tabs = [build_tables(s) for s in specs]
    meshes = [capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) for t in tabs]
    try:
        with capi.GpuBatch(meshes) as b:
            b.run(23, sync=False)  # no batch_synchronize before the read-back
            got = [fetch(capi._lib, g.h, "tlm_gpu_fetch_links_noalloc", (t["nz"], t["ny"], t["nx"], 12))
                   for g, t in zip(meshes, tabs)]
            again = fetch(capi._lib, meshes[0].h, "tlm_gpu_fetch_links_noalloc",
                          (tabs[0]["nz"], tabs[0]["ny"], tabs[0]["nx"], 12))
            b.synchronize()
            ref = [g.links() for g in meshes]
        for a, r in zip(got + [again], ref + [ref[0]]):
            scale = np.max(np.abs(r))
            assert scale > 0
            assert np.max(np.abs(a - r)) <= TOL * scale
    finally:
        for g in meshes:
            g.close()


def test_noalloc_fetch_rejects_oversized_mesh(gpu_lib):
    t = build_tables(cases.pec_box(n=45, steps=3))  # 91125 cells > 87381
    with capi.GpuMesh(t) as g:
        g.run(1)
        with pytest.raises(capi.TLMError) as e:
            fetch(capi._lib, g.h, "tlm_gpu_fetch_links_noalloc", (45, 45, 45, 12))
        assert e.value.code == -1 and "limit" in str(e.value)


def test_noalloc_fetch_needs_device_state(gpu_lib):
    t = build_tables(cases.pec_box(n=8, steps=3))
    with capi.GpuMesh(t) as g:
        with pytest.raises(capi.TLMError) as e:
            fetch(capi._lib, g.h, "tlm_gpu_fetch_links_noalloc", (8, 8, 8, 12))
        assert e.value.code == -5
