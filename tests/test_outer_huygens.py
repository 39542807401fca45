"""Huygens surface on the outer boundary (huygens_surface.F90:508-612,
TLM_SOLVER/outer_boundary.F90:133-318).

Physical pin: a 20^3 box whose outer boundary launches the plane wave of
TEST_DATA/HUYGENS_SURFACE must see at its centre what the reference saw
inside its closed 20^3-cell Huygens box embedded in a 40^3 mesh (the golden
series), up to the field that box let outside.  The GPU path is checked
against the oracle.
"""
import os

import numpy as np
import pytest

from ggi_tlm_b200 import capi, cases
from ggi_tlm_b200.problem import HuygensOuter, OutputPoint, ProblemSpec, build_tables, probe_series

import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def spec(component="Ex", R=0.0):
    big = cases.kat_huygens_box(component)
    return ProblemSpec(nx=20, ny=20, nz=20, dl=big.dl, n_timesteps=big.n_timesteps, R=(R,) * 6, origin=(-1.0,) * 3,
                       functions=big.functions, huygens=HuygensOuter(1, 54.73, 45.0, 1.0, 0.5),
                       outputs=[OutputPoint((11, 11, 11), component), OutputPoint((4, 15, 9), "Hy")])


@pytest.mark.parametrize("component", ["Ex", "Ey", "Ez", "Hx", "Hy", "Hz"])
def test_oracle_outer_huygens_launches_the_golden_plane_wave(component):
    t = build_tables(spec(component))
    assert t["hs_n"] == 6 * 20 * 20 and t["n_faces"] == 0
    p = probe_series(t, O.Oracle(t).run(t["n_timesteps"]))[0]
    g = np.load(os.path.join(GOLDEN, f"huygens_box_{component}.npz"))["value"]
    assert np.linalg.norm(p - g) / np.linalg.norm(g) < 2e-3  # measured 4.8e-4 (Ex, Hz)


def test_oracle_outer_huygens_sign_matters():
    t = build_tables(spec())
    t["hs_Hi"] = -np.asarray(t["hs_Hi"])  # the wrong H: no clean plane wave inside
    p = probe_series(t, O.Oracle(t).run(t["n_timesteps"]))[0]
    g = np.load(os.path.join(GOLDEN, "huygens_box_Ex.npz"))["value"]
    assert np.linalg.norm(p - g) / np.linalg.norm(g) > 0.1


@pytest.mark.gpu
@pytest.mark.parametrize("R", [0.0, -0.5])
def test_gpu_outer_huygens_matches_oracle(gpu_lib, R):
    t = build_tables(spec("Ez", R))
    o = O.Oracle(t)
    po = probe_series(t, o.run(t["n_timesteps"]))
    lo = o.links()
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.run(50)
        g.run(t["n_timesteps"] - 50)
        pg = probe_series(t, g.cell_output())
        lg = g.links()
    for i in range(len(po)):
        assert np.linalg.norm(pg[i] - po[i]) <= 1e-10 * np.linalg.norm(po[i])
    assert np.abs(lg - lo).max() <= 1e-10 * np.abs(lo).max()
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP32) as g:
        g.run(t["n_timesteps"])
        p32 = probe_series(t, g.cell_output())
    for i in range(len(po)):
        assert np.linalg.norm(p32[i] - po[i]) <= 1e-4 * np.linalg.norm(po[i])


@pytest.mark.gpu
def test_gpu_outer_huygens_in_a_batch_equals_solo(gpu_lib):
    tabs = [build_tables(spec("Ex")), build_tables(spec("Hz", -0.3)),
            build_tables(cases.pml_spheres(n=20, pml=4, n_spheres=2, steps=90, n_probes=3, n_freq=2, dft_size=6,
                                           rmin=2, rmax=3))]
    solo = []
    for t in tabs:
        with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
            g.set_variant(1)
            g.run(t["n_timesteps"])
            solo.append(g.cell_output())
    meshes = [capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) for t in tabs]
    with capi.GpuBatch(meshes) as b:
        b.set_variant(1)
        b.run(1000)
    for g, co in zip(meshes, solo):
        assert np.array_equal(g.cell_output(), co)
        g.close()
