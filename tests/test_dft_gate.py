"""Output steps of frequency-domain output surfaces: a surface's DFT takes
only the timesteps first..last every interval (get_output_flag,
OUTPUT/output.F90:564-598, applied in face_output_frequency_output_surfaces,
frequency_output_surfaces.F90:336-342).

CPU: the reader keeps the surface's output_timestep_information block; on
the oracle a gate over every step changes nothing (bit for bit), and the
odd-step and even-step gates add up to the ungated transform.  GPU: the
library's gated transform against the oracle's."""
import dataclasses
import os
import sys

import numpy as np
import pytest

from ggi_tlm_b200.problem import build_tables

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import test_inp as T  # noqa: E402
import oracle  # noqa: E402

GATED = T.ALL_OUTPUTS.replace("2e8\nJx\n", "2e8\nJx\noutput_timestep_information\n2\n30\n3\n")


def spec_with(**gate):
    s = T.small(base=T.ALL_OUTPUTS).spec
    s.dft_surfaces = [dataclasses.replace(d, **gate) for d in s.dft_surfaces]
    return s


def dft_of(spec):
    t = build_tables(spec)
    o = oracle.Oracle(t)
    o.run(int(t["n_timesteps"]))
    d = o.dft()
    o.close()
    return d


def test_reader_keeps_the_surface_output_steps():
    s = T.small(base=GATED).spec
    ds = s.dft_surfaces[0]
    assert (ds.first_step, ds.last_step, ds.interval) == (2, 30, 3)
    t = build_tables(s)
    assert (list(t["dft_first"]), list(t["dft_last"]), list(t["dft_interval"])) == ([2], [30], [3])
    ungated = build_tables(T.small(base=T.ALL_OUTPUTS).spec)
    assert list(ungated["dft_last"]) == [int(ungated["n_timesteps"])]


def test_oracle_gates_add_up():
    n = int(T.small(base=T.ALL_OUTPUTS).spec.n_timesteps)
    full = dft_of(spec_with())
    assert np.abs(full).max() > 0
    np.testing.assert_array_equal(dft_of(spec_with(first_step=1, last_step=n, interval=1)), full)
    odd = dft_of(spec_with(first_step=1, interval=2))
    even = dft_of(spec_with(first_step=2, interval=2))
    assert np.linalg.norm(odd + even - full) <= 1e-12 * np.linalg.norm(full)
    assert np.linalg.norm(odd - full) > 1e-3 * np.linalg.norm(full)
    window = dft_of(spec_with(first_step=2, last_step=30, interval=3))
    assert np.linalg.norm(window - full) > 1e-3 * np.linalg.norm(full)


@pytest.mark.gpu
def test_gpu_gated_dft_matches_the_oracle(gpu_lib):
    from ggi_tlm_b200 import capi

    t = build_tables(T.small(base=GATED).spec)
    o = oracle.Oracle(t)
    o.run(int(t["n_timesteps"]))
    want = o.dft()
    o.close()
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.run(int(t["n_timesteps"]))
        got = g.dft()
    assert got.shape == want.shape
    assert np.linalg.norm(got - want) <= 1e-10 * np.linalg.norm(want)
