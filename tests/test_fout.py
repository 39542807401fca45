"""Frequency-domain results (ggi_tlm_b200/fout.py) against the reference's
own golden spectra (tests/golden/fout_text.npz, by tests/golden/make_golden.py).

The reference's CAVITY_FREE_SPACE, CAVITY_EPSR=2, CAVITY_MUR=2 and
PARALLEL_TEST cases are read from their own .inp files
(tests/golden/inp_text.npz), run, written as .field.tout (E16.7, as the
reference prints them), and Fourier transformed as their post-processing
recipe asks (option 3: point 1, lin 1 MHz to 300 MHz, 1000 frequencies;
100 for PARALLEL_TEST).  The spectra must equal the golden .fout_ref files
to their print precision.  CPU: through the oracle, and the .fout writer
on the golden lines.  GPU: the same through the library in FP64."""
import os
import sys

import numpy as np
import pytest

from ggi_tlm_b200 import capi, fout, tout
from ggi_tlm_b200.inp import read_inp, read_inp_lenient
from ggi_tlm_b200.problem import build_tables, probe_series

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import oracle  # noqa: E402
import test_inp  # noqa: E402

CASES = {"cavity_free_space": 1000, "cavity_epsr2": 1000, "cavity_mur2": 1000, "parallel_test": 100}
TOL = 5e-7  # relative L2 of the complex spectrum: the E16.7 print precision of both files


def golden(name):
    d = np.load(os.path.join(HERE, "golden", "fout_text.npz"))
    return [str(x) for x in d[name]]


def problem(name):
    p = read_inp(test_inp.inputs()[name], test_inp.materials)
    return p, build_tables(p.spec)


def spectrum(p, t, cell_out, face_out, n_freq):
    """The post-processing recipe on the .field.tout text the run writes."""
    rows = tout.field_rows(t, probe_series(t, cell_out), face_out, timing=p.output_timing)
    text = tout.format_rows(rows)
    printed = np.array([[float(x[:16]), int(x[16:21]), float(x[21:])] for x in text])
    time, value = fout.tout_series(printed, 1)
    freqs = fout.frequencies(1e6, 3e8, n_freq)
    return freqs, fout.fourier_transform(time, value, freqs)


def check(name, freqs, v):
    g = fout.read_fout(golden(name))
    assert g.shape == (len(freqs), 7)
    np.testing.assert_allclose(freqs, g[:, 0], rtol=5.01e-7)
    gv = g[:, 2] + 1j * g[:, 3]
    assert np.linalg.norm(v - gv) / np.linalg.norm(gv) < TOL, name
    # the resonances: |V| and dB where the spectrum is within 20 dB of its peak
    big = np.abs(gv) > 0.1 * np.abs(gv).max()
    np.testing.assert_allclose(np.abs(v[big]), g[big, 4], rtol=2e-6)
    np.testing.assert_allclose(20 * np.log10(np.abs(v[big])), g[big, 6], atol=1e-4)


def test_fout_writer_on_the_golden_lines():
    for name in CASES:
        lines = golden(name)
        g = fout.read_fout(lines)
        assert lines[:3] == fout.header(1, len(g))
        for row, line in zip(g, lines[3:]):
            mine = fout.data_line(row[0], int(row[1]), complex(row[2], row[3]))
            assert mine[:53] == line[:53]  # f, point, Re, Im as printed
            # |V|, phase and dB from the printed Re, Im: within a unit or two of the last digit
            np.testing.assert_allclose([float(mine[53 + 16 * k:69 + 16 * k]) for k in range(3)], row[4:7],
                                       rtol=3e-6, atol=1e-12)


def test_frequency_grids():
    f = fout.frequencies(1e6, 3e8, 1000)
    assert f[0] == 1e6 and abs(f[-1] - 3e8) < 1e-6 and len(f) == 1000
    lg = fout.frequencies(1e6, 1e9, 4, "log")
    np.testing.assert_allclose(lg, [1e6, 1e7, 1e8, 1e9], rtol=1e-14)
    assert list(fout.frequencies(5e6, 9e6, 1)) == [5e6]
    with pytest.raises(ValueError):
        fout.frequencies(1, 2, 3, "octave")


def test_transform_of_a_known_signal():
    """A decaying exponential exp(-a t) sampled every dt transforms to the
    geometric sum dt / (1 - exp(-(a + j w) dt)) (for many steps)."""
    dt, a, n = 1e-10, 2e8, 4000
    time = np.arange(n) * dt
    freqs = np.array([0.0, 1e8, 3e8])
    v = fout.fourier_transform(time, np.exp(-a * time), freqs)
    want = dt / (1 - np.exp(-(a + 2j * np.pi * freqs) * dt))
    np.testing.assert_allclose(v, want, rtol=1e-12)


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_spectra_match_reference_golden(name):
    p, t = problem(name)
    o = oracle.Oracle(t)
    cell = o.run(t["n_timesteps"])
    face = o.face_probes() if int(t["n_face_probes"]) else np.zeros((0, t["n_timesteps"]))
    check(name, *spectrum(p, t, cell, face, CASES[name]))


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_spectra_match_reference_golden(gpu_lib, name):
    p, t = problem(name)
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.run(t["n_timesteps"])
        cell, face = g.cell_output(), g.face_output()
    check(name, *spectrum(p, t, cell, face, CASES[name]))


def test_command_line_transform(tmp_path):
    """.tout -> .fout from the command line equals the in-process transform."""
    p, t = problem("parallel_test")
    o = oracle.Oracle(t)
    cell = o.run(t["n_timesteps"])
    src = str(tmp_path / "cavity.field.tout")
    tout.write_tout(src, tout.field_rows(t, probe_series(t, cell), np.zeros((0, t["n_timesteps"]))), 1,
                    t["n_timesteps"])
    out = str(tmp_path / "cavity.fout")
    assert fout.main([src, "1", "lin", "1e6", "3e8", "100", out]) == 0
    with open(out) as f:
        lines = f.read().splitlines()
    freqs, v = spectrum(p, t, cell, np.zeros((0, t["n_timesteps"])), 100)
    assert lines == fout.format_fout(freqs, v)
    check("parallel_test", freqs, v)
    assert fout.main([src, "7", "lin", "1e6", "3e8", "100", out]) == 1  # no such point


def shielding_effectiveness(p, t, cell_out, face_out):
    """SHIELDING_EFFECTIVENESS_BOX_SLOT's recipe: option 3 on box_slot.excitation.tout
    and on box_slot.field.tout (point 1, lin 1 MHz to 300 MHz, 1000
    frequencies), each written as .fout and read back, then option 6 with
    A = B = 1, C = 0: excitation / Ey."""
    freqs = fout.frequencies(1e6, 3e8, 1000)
    spectra = []
    files = [(tout.excitation_rows(t), False),  # the excitation file is written without the 1e-30 flush
             (tout.field_rows(t, probe_series(t, cell_out), face_out, timing=p.output_timing), True)]
    for rows, flush in files:
        printed = [tout.data_line(*r, flush_small=flush) for r in rows]
        series = np.array([[float(x[:16]), int(x[16:21]), float(x[21:])] for x in printed])
        v = fout.fourier_transform(*fout.tout_series(series, 1), freqs)
        spectra.append(fout.spectrum(fout.read_fout(fout.format_fout(freqs, v)))[1])
    return freqs, fout.combine(spectra[0], spectra[1], 1.0, 1.0, 0.0)


def test_oracle_shielding_effectiveness_matches_reference_golden():
    """A PEC box with a free-space slot in its top face (the slot's surface
    material overrides the box's), lit by a plane wave from the outer
    Huygens surface, 29979 steps."""
    p, t = problem("box_slot")
    assert [sh.kind for sh in p.spec.surface_sheets] == ["PEC"] * 6 + ["free"]
    o = oracle.Oracle(t)
    cell = o.run(t["n_timesteps"])
    check("box_slot", *shielding_effectiveness(p, t, cell, np.zeros((0, t["n_timesteps"]))))


@pytest.mark.gpu
def test_gpu_shielding_effectiveness_matches_reference_golden(gpu_lib):
    p, t = problem("box_slot")
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.run(t["n_timesteps"])
        cell = g.cell_output()
    check("box_slot", *shielding_effectiveness(p, t, cell, np.zeros((0, t["n_timesteps"]))))


def power_calc():
    p = read_inp_lenient(test_inp.inputs()["power_calc"], test_inp.materials)
    return p, build_tables(p.spec)


def check_power_calc(t, face, acc):
    """POWER_CALCS: an impulse plane wave from the outer Huygens surface.  The
    zmax-face probe against power_calc.field.tout_ref, and the power through
    a 1 m^2 patch against power_calc.frequency_domain_power_surface.fout_ref.
    That file predates the removal of the dt factor from the power
    accumulators (frequency_domain_power_surfaces.F90:331, "remove dt
    normalisation here"), which this library follows, so it is compared
    with P dt^2."""
    g = np.load(os.path.join(HERE, "golden", "power_calc_Ex.npz"))["value"]
    v = np.where(np.abs(face[0]) < 1e-30, 0.0, face[0])
    assert np.linalg.norm(v - g) / np.linalg.norm(g) < TOL
    power = fout.power_surfaces(t, acc)
    lines = fout.power_surface_lines(t["ps_freq"], [1] * len(power), power)
    gl = golden("power_calc")
    assert lines[:3] == gl[:3] and len(lines) == len(gl)
    gf = fout.read_fout(gl)
    np.testing.assert_allclose(np.asarray(t["ps_freq"]), gf[:, 0], rtol=5.01e-7)
    scaled = power * float(t["dt"]) ** 2
    assert np.linalg.norm(scaled.real - gf[:, 2]) / np.linalg.norm(gf[:, 2]) < TOL
    assert np.abs(scaled.imag - gf[:, 3]).max() < 1e-9 * np.abs(gf[:, 2]).max()


def test_oracle_power_calcs_matches_reference_golden():
    p, t = power_calc()
    assert p.skipped == ["output_surface_list: an output surface on a rotated rectangle: only zero Euler angles "
                         "are supported"]
    o = oracle.Oracle(t)
    o.run(t["n_timesteps"])
    check_power_calc(t, o.face_probes(), oracle.power_surfaces(t))


@pytest.mark.gpu
def test_gpu_power_calcs_matches_reference_golden(gpu_lib):
    p, t = power_calc()
    with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64) as g:
        g.run(t["n_timesteps"])
        face, acc = g.face_output(), g.power_surfaces()
    check_power_calc(t, face, acc)


def test_transmission_cross_section_reproduces_the_reference_file():
    """POWER_CALCS's TCS.fout_ref (post-processor option 15), byte for byte:
    the transmitted power from the case's golden power surface file over the
    spectrum of its golden field series (option 3, 1 .. 600 MHz, 100
    frequencies, as its post-processing input asks)."""
    from ggi_tlm_b200 import fout

    d = np.load(os.path.join(HERE, "golden", "fout_text.npz"))
    g = np.load(os.path.join(HERE, "golden", "power_calc_Ex.npz"))
    freqs = fout.frequencies(1e6, 600e6, 100, "lin")
    sel = g["point"] == 1
    field = fout.read_fout(fout.format_fout(freqs, fout.fourier_transform(g["time"][sel], g["value"][sel], freqs)))
    power = fout.read_fout([str(x) for x in d["power_calc"]])
    assert fout.transmission_cross_section_lines(power, field, "e") == [str(x) for x in d["power_calc_tcs"]]


def test_oneport_analysis_recovers_a_known_wave():
    """Post-processor option 9 on the fields of one known wave in a uniform
    section: E = a exp(-j beta x) + b exp(j beta x), H = (a exp(-j beta x) -
    b exp(j beta x)) / Z on planes at x = -d, +d; the analysis returns beta,
    Z and R = (b / a) exp(2 j beta l), the reflection at x = l."""
    from ggi_tlm_b200 import fout

    freqs = np.array([1e9, 5e9, 2e10])
    d_port, l, z = 0.2e-3, 2.5e-3, 300.0 + 20.0j
    beta = 2 * np.pi * freqs / 2.9e8 * (1.0 - 0.01j) * 1.3
    a, b = 1.0 + 0.0j, 0.4 * np.exp(0.3j)
    P = np.exp(1j * beta * d_port / 2)
    ft = [a * P + b / P, a / P + b * P, (a * P - b / P) / z, (a / P - b * P) / z]
    lines, zs_lines = fout.oneport_lines(freqs, ft, d_port, l)
    assert lines[0].split()[:3] == ["frequency", "Re{Beta}", "Im{Beta}"] and len(lines) == 4 and len(zs_lines) == 4
    rows = np.loadtxt(lines[1:])
    r = b / a * np.exp(2j * beta * l)
    want = np.column_stack([freqs, beta.real, beta.imag, np.full(3, z.real), np.full(3, z.imag), r.real, r.imag,
                            np.abs(r), 20 * np.log10(np.abs(r)), (2 * np.pi * freqs / beta).real, 1 - np.abs(r) ** 2])
    np.testing.assert_allclose(rows, want, rtol=1e-4, atol=1e-9)
    zs = np.loadtxt(zs_lines[1:])
    np.testing.assert_allclose(zs[:, 1] + 1j * zs[:, 2], z * (1 + r) / (1 - r), rtol=1e-4)
