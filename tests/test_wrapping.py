"""Wrapping boundaries (Wrapping_boundary_conditions; wrap_outer_boundary,
TLM_SOLVER/wrap_outer_boundary.F90:101-273): the two outer faces of a
wrapped axis are joined, each boundary port receiving R times the reflected
pulse of the cell at the other end.

CPU: the reference's WRAPPING_BOUNDARY case read from its own input file
reproduces its golden series on the oracle (and not without the wrap).
GPU: the library against the oracle, all axes and one axis at a time, in
FP64 and through the bulk kernel variants."""
import os
import sys

import numpy as np
import pytest

from ggi_tlm_b200 import capi, cases, inp
from ggi_tlm_b200.problem import HuygensOuter, UnsupportedFeature, build_tables, probe_series

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import test_inp as T  # noqa: E402
import oracle  # noqa: E402


def wrapping_case():
    return inp.read_inp(T.inputs()["wrapping"], T.materials)


def test_reader_takes_the_flags():
    p = wrapping_case()
    assert p.spec.wrap == (1, 1, 1) and p.skipped == []
    assert list(build_tables(p.spec)["wrap"]) == [1, 1, 1]
    bad = T.BASE + "Wrapping_boundary_conditions\n1 2 0\n"
    with pytest.raises(ValueError, match="1 or 0"):
        inp.read_inp(bad.splitlines(), T.materials)


@pytest.mark.parametrize("wrap", [(1, 1, 1), (0, 0, 0)])
def test_oracle_matches_the_reference_wrapping_case(wrap):
    p = wrapping_case()
    p.spec.wrap = wrap
    t = build_tables(p.spec)
    v = probe_series(t, oracle.Oracle(t).run(t["n_timesteps"]))[0]
    v = np.where(np.abs(v) < 1e-30, 0.0, v)
    g = np.load(os.path.join(HERE, "golden", "wrapping_Ex.npz"))["value"]
    rel = np.linalg.norm(v - g) / np.linalg.norm(g)
    if wrap == (1, 1, 1):
        assert rel < 5e-7
    else:  # the golden series really pins the wrap
        assert rel > 5e-3


def test_outer_huygens_with_wrap_is_refused():
    s = cases.pec_box(n=10, steps=5)
    s.huygens = HuygensOuter(1, 0.0, 0.0, 1.0, 0.0)
    s.wrap = (1, 0, 0)
    with pytest.raises(UnsupportedFeature, match="wrapping"):
        build_tables(s)


def ragged(wrap):
    s = cases.pml_spheres(n=20, pml=0, n_spheres=2, steps=60, n_probes=4, n_freq=2, dft_size=4, rmin=2.0, rmax=3.0)
    s.nx, s.ny, s.nz = 21, 22, 23
    s.R = (-1.0, 0.5, 1.0, -0.3, 0.2, 0.0)
    s.wrap = wrap
    return s


@pytest.mark.gpu
@pytest.mark.parametrize("wrap", [(1, 1, 1), (1, 0, 0), (0, 1, 0), (0, 0, 1)])
def test_gpu_wrapping_matches_the_oracle(gpu_lib, wrap):
    t = build_tables(ragged(wrap)) if wrap != (1, 1, 1) else build_tables(wrapping_case().spec)
    o = oracle.Oracle(t)
    want = o.run(t["n_timesteps"])
    wl = o.links()
    o.close()
    for variant in range(capi.num_variants()):
        with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
            g.set_variant(variant)
            g.run(t["n_timesteps"])
            got, links = g.cell_output(), g.links()
        assert got.shape == want.shape
        assert np.linalg.norm(got - want) <= 1e-10 * np.linalg.norm(want), variant
        assert np.linalg.norm(links - wl) <= 1e-10 * np.linalg.norm(wl), variant
