"""Excitation function tables (problem.excitation_tables, restating
EXCITATION/excitation.F90:155-559) for the types no golden series covers,
checked against the properties the reference's formulas state: peak
normalisation of the differential Gaussian and the double exponential, the
envelopes of the stepped and pulsed sinusoids, and the reference's face
value of the double exponential and ring wave, which takes 1/amplitude."""
import math

import numpy as np
import pytest

from ggi_tlm_b200.inp import read_inp
from ggi_tlm_b200.problem import ExcitationFunction, build_tables, excitation_tables

DT = 1e-12
N = 20000


def table(kind, params):
    return excitation_tables([ExcitationFunction(kind, tuple(params))], N, DT)


def times():
    t = np.arange(N) * DT
    return t, t + DT / 2


def test_differential_gaussian_peaks_at_its_amplitude():
    amp, width, delay = 3.0, 0.5e-9, 5e-9
    val, valf = table("differential_gaussian", (amp, width, delay))
    assert abs(val.max() - amp) < 1e-5 * amp and abs(val.min() + amp) < 1e-5 * amp
    t, _ = times()
    assert t[val[0].argmax()] == pytest.approx(delay - width / math.sqrt(2), abs=2 * DT)
    assert np.all(val[0][np.abs(t - delay) >= 5 * width] == 0.0)


def test_double_exponential_and_ring_wave():
    amp, tau1, tau2, f = 2.0, 2e-9, 0.2e-9, 1e9
    val, valf = table("double_exponential", (amp, tau1, tau2))
    assert abs(val.max() - amp) < 1e-6 * amp  # normalised by its value at tpeak
    t, t2 = times()
    alpha, beta = 1 / tau1, 1 / tau2
    tpeak = (math.log(beta) - math.log(alpha)) / (beta - alpha)
    fpeak = math.exp(-alpha * tpeak) - math.exp(-beta * tpeak)
    # the face values use 1/amplitude (excitation.F90:385-393)
    np.testing.assert_allclose(valf[0], (1 / amp / fpeak) * (np.exp(-alpha * t2) - np.exp(-beta * t2)), rtol=1e-12)
    rv, rvf = table("ring_wave", (amp, tau1, tau2, f))
    np.testing.assert_allclose(rv[0], val[0] * np.sin(2 * math.pi * f * t), rtol=1e-12, atol=1e-300)
    np.testing.assert_allclose(rvf[0], valf[0] * np.sin(2 * math.pi * f * t2), rtol=1e-12, atol=1e-300)


def test_gaussian_step_sinusoid_and_sinusoidal_pulse():
    amp, width, delay, f, ph = 1.5, 1e-9, 6e-9, 2e9, 30.0
    val, _ = table("gaussian_step_sinusoid", (amp, width, delay, f, ph))
    t, _ = times()
    after = t >= delay
    np.testing.assert_allclose(val[0][after], amp * np.sin(2 * math.pi * f * t[after] - ph * math.pi / 180), rtol=1e-12)
    assert np.all(val[0][t < delay - 5 * width] == 0.0)
    t1, t2, t3, t4 = 2e-9, 4e-9, 10e-9, 14e-9
    pv, _ = table("sinusoidal_pulse", (amp, f, ph, t1, t2, t3, t4))
    s = amp * np.sin(2 * math.pi * f * t - ph * math.pi / 180)
    flat = (t >= t2) & (t <= t3)
    np.testing.assert_allclose(pv[0][flat], s[flat], rtol=1e-12)
    assert np.all(pv[0][(t < t1) | (t > t4)] == 0.0)
    ramp = (t >= t1) & (t < t2)
    np.testing.assert_allclose(pv[0][ramp], s[ramp] * (t[ramp] - t1) / (t2 - t1), rtol=1e-12, atol=1e-300)


def test_reader_takes_the_new_types():
    text = """Mesh_outer_boundary_dimension
0 1 0 1 0 1
Mesh_cell_dimension
0.1
Excitation_function_list
4
1
gaussian_step_sinusoid
1.0 1e-9 3e-9 1e9 0.0
2
double_exponential
1.0 2e-9 0.2e-9
3
sinusoidal_pulse
1.0 1e9 0.0 1e-9 2e-9 3e-9 4e-9
4
ring_wave
1.0 2e-9 0.2e-9 1e9
Simulation_time
1e-8
"""
    p = read_inp(text.splitlines(), lambda name: None)
    assert [f.type for f in p.spec.functions] == ["gaussian_step_sinusoid", "double_exponential",
                                                  "sinusoidal_pulse", "ring_wave"]
    t = build_tables(p.spec)
    assert np.asarray(t["fn_value"]).reshape(4, -1).shape[1] == t["n_timesteps"]
