"""FP64 GPU parity at the benchmarked sizes.

The 256^3 PML-spheres mesh (8-cell PML, 32 dielectric spheres, Huygens plane
wave, 16 probes, 64 frequencies x 64 x 64 DFT faces) and the 384x384x192
Debye-slab mesh (10-cell PML, 6 two-pole Debye slabs, 64 x 64 DFT) are run
for a few dozen steps on the GPU and on the oracle (its z-planes shared
among the host's threads; bit-identical to one thread) from the same
tables, and compared: every probe sample, the DFT accumulators and the
complete link state.  At these sizes the tile lists, the PML shell decoder
at 8 and 10 cells, the special-cell lists and the step graphs are the ones
the benchmark runs."""
import os

import numpy as np
import pytest

from ggi_tlm_b200 import capi, cases
from ggi_tlm_b200.problem import build_tables

import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def _rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / nb if nb > 0 else np.linalg.norm(a)


def _links_rel(a, b):
    """Relative L2 of two link states, summed plane by plane (no full-size temporaries)."""
    num = den = 0.0
    for z in range(a.shape[0]):
        d = a[z] - b[z]
        num += float(np.dot(d.ravel(), d.ravel()))
        den += float(np.dot(b[z].ravel(), b[z].ravel()))
    return np.sqrt(num / den) if den > 0 else np.sqrt(num)


def _compare(t, steps):
    o = O.Oracle(t, threads=_threads())
    want = o.run(steps)
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.run(steps)
        got, dft, links = g.cell_output(1, steps), g.dft(), g.links()
    wl = o.links()
    assert np.any(wl != 0.0)
    assert _links_rel(links, wl) <= TOL
    del links
    assert got.shape == want.shape
    assert _rel(got, want) <= TOL or np.array_equal(got, want)
    wd = o.dft()
    assert dft.shape == wd.shape
    assert _rel(dft, wd) <= TOL or np.array_equal(dft, wd)
    o.close()


def test_gpu_fp64_pml_spheres_256_full_size(gpu_lib):
    t = build_tables(cases.pml_spheres())
    assert (t["nx"], t["ny"], t["nz"]) == (256, 256, 256) and int(t["dft_face_ptr"][-1]) == 64 * 64 * 64
    _compare(t, 24)


def test_gpu_fp64_debye_slabs_384x384x192_full_size(gpu_lib):
    t = build_tables(cases.debye_slabs())
    assert (t["nx"], t["ny"], t["nz"]) == (384, 384, 192)
    assert int((np.asarray(t["mat_eps_order"]) == 3).sum()) == 6
    _compare(t, 24)
