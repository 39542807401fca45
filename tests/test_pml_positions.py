"""PML cell positions: the kernels decode them from the PML number when the
PML cells form the usual box shell, and load them from the position list
otherwise (forced here with TLM_PML_SHELL=0).  Both give identical results,
on meshes with unequal PML thicknesses per face, PML probes and PML cells in
a material."""
import os

import numpy as np
import pytest

from ggi_tlm_b200 import capi, cases
from ggi_tlm_b200.problem import OutputPoint, build_tables

pytestmark = pytest.mark.gpu


def shells():
    a = cases.pml_spheres(n=26, pml=4, n_spheres=2, steps=60, n_probes=3, n_freq=2, dft_size=6, rmin=2, rmax=3)
    a.pml_cells = (3, 5, 0, 4, 2, 6)          # unequal, one face without PML
    a.outputs += [OutputPoint((2, 10, 10), "Ez"), OutputPoint((24, 3, 25), "Hx")]  # probes inside the PML
    b = cases.pml_dielectric_slab(28, 6, 60, slab_top=10)  # PML cells in a material
    c = cases.pml_point_source(14, 40, 30, pml=5, steps=60)  # thin in x
    return [build_tables(s) for s in (a, b, c)]


def run(t, precision):
    with capi.GpuMesh(t, precision=precision) as g:
        g.run(t["n_timesteps"])
        return g.cell_output(), g.links()


@pytest.mark.parametrize("precision", [capi.TLM_PRECISION_FP32, capi.TLM_PRECISION_FP64])
def test_shell_decode_equals_position_list(gpu_lib, precision):
    for t in shells():
        os.environ.pop("TLM_PML_SHELL", None)
        a = run(t, precision)
        os.environ["TLM_PML_SHELL"] = "0"
        try:
            b = run(t, precision)
        finally:
            os.environ.pop("TLM_PML_SHELL", None)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
