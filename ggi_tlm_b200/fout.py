"""Frequency-domain result files in the reference's text format, and the
post-processor's Fourier transform that makes them from a .tout series.

GGI_TLM_post_process option 3 (POST_PROCESSOR/fourier_transform.F90)
reads one output point's series from a .tout file
(read_write_time_domain_data.F90:36-223: the rows whose point number
matches, times and values as printed), takes dt as the difference of the
first two printed times, and evaluates at each frequency of a linear or
logarithmic grid the sum  V(f) = sum_k v_k exp(-j 2 pi f t_k) dt  in step
order.  write_frequency_domain_data (read_write_frequency_domain_data.F90:
38-83) writes a three-line header and one ``(E16.7,I5,5E16.7)`` line per
frequency: f, the point number 1, Re V, Im V, |V|, atan2(Im, Re) and
20 log10 |V|.  Option 10 (two-port analysis, ``twoport_lines``) turns the
spectra of two planes on each side of a scatterer into S-parameters.
"""
from __future__ import annotations

import cmath
import math
from typing import List, Sequence, Tuple

import numpy as np

from .problem import Z0
from .tout import fortran_e

HEADER = "# Frequency Domain Data"  # frequency_domain_output_file_header


def header(n_points: int, n_frequencies: int) -> List[str]:
    """write_frequency_domain_header_data: the title and two ``(A25,I10)`` counts."""
    return [HEADER, "# Number of data points: " + f"{n_points:10d}",
            "# Number of frequencies: " + f"{n_frequencies:10d}"]


def frequencies(fmin: float, fmax: float, n: int, scale: str = "lin") -> np.ndarray:
    """The frequency grid of fourier_transform.F90: fmin + (k-1) fstep, or
    10**(log10 fmin + (k-1) log_fstep) for a log scale."""
    if scale == "log":
        lo, hi = math.log10(fmin), math.log10(fmax)
        step = (hi - lo) / float(n - 1) if n != 1 else 0.0
        return np.array([10.0 ** (lo + (k - 1) * step) for k in range(1, n + 1)])
    if scale != "lin":
        raise ValueError(f"frequency scale {scale!r}: lin or log")
    step = (fmax - fmin) / float(n - 1) if n != 1 else 0.0
    return np.array([fmin + (k - 1) * step for k in range(1, n + 1)])


def fourier_transform(time: np.ndarray, value: np.ndarray, freqs: np.ndarray) -> np.ndarray:
    """V(f) = sum_k value_k exp(-j 2 pi f time_k) dt with dt = time[1] - time[0],
    summed in step order for every frequency at once."""
    time = np.asarray(time, dtype=np.float64)
    value = np.asarray(value, dtype=np.float64)
    dt = time[1] - time[0]
    w = 2.0 * math.pi * np.asarray(freqs, dtype=np.float64)
    acc = np.zeros(w.shape, dtype=np.complex128)
    for t, v in zip(time, value):
        acc = acc + v * np.exp(-1j * w * t) * dt
    return acc


def data_line(f: float, point: int, v: complex) -> str:
    mag = abs(v)
    db = 20.0 * math.log10(mag) if mag > 0.0 else -math.inf
    fields = [v.real, v.imag, mag, math.atan2(v.imag, v.real), db]
    return fortran_e(f) + f"{int(point):5d}" + "".join(fortran_e(x) for x in fields)


def format_fout(freqs: Sequence[float], values: Sequence[complex], point: int = 1) -> List[str]:
    """The lines of a one-point .fout file."""
    return header(1, len(freqs)) + [data_line(f, point, complex(v)) for f, v in zip(freqs, values)]


def write_fout(path: str, freqs: Sequence[float], values: Sequence[complex], point: int = 1) -> None:
    with open(path, "w") as f:
        for line in format_fout(freqs, values, point):
            f.write(line + "\n")


def read_fout(path_or_lines) -> np.ndarray:
    """The numeric rows of a .fout file, [n, 7]."""
    if isinstance(path_or_lines, str):
        return np.loadtxt(path_or_lines, comments="#", ndmin=2)
    return np.loadtxt([x for x in path_or_lines if not x.startswith("#")], ndmin=2)


def spectrum(rows: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """(frequencies, complex values) of .fout rows [n, 7] (read_fout), as
    read_frequency_domain_data takes them
    (POST_PROCESSOR/read_write_frequency_domain_data.F90:155-260): from the
    printed Re and Im columns through CMPLX() without a kind, i.e. rounded
    to single precision."""
    re = rows[:, 2].astype(np.float32).astype(np.float64)
    im = rows[:, 3].astype(np.float32).astype(np.float64)
    return rows[:, 0], re + 1j * im


def combine(f1: np.ndarray, f2: np.ndarray, a: float = 1.0, b: float = 1.0, c: float = 0.0) -> np.ndarray:
    """Post-processor option 6 (POST_PROCESSOR/combine_frequency_domain_data.F90):
    (A f1) / (B f2) + C at each frequency; the two grids must be equal."""
    return (a * np.asarray(f1)) / (b * np.asarray(f2)) + c


def tout_series(rows: np.ndarray, point: int) -> Tuple[np.ndarray, np.ndarray]:
    """(time, value) of one output point from .tout rows [n, 3] (read_tout)."""
    sel = rows[:, 1] == point
    return rows[sel, 0], rows[sel, 2]


def power_surfaces(tables: dict, acc: np.ndarray) -> np.ndarray:
    """write_frequency_domain_power_surfaces (OUTPUT/frequency_domain_power_surfaces.F90:
    420-574): per power surface entry (surface, frequency) the sum over its
    faces of sign (E1 H2* - E2 H1*) dl^2 / 2, sign +1 on a min face and -1 on
    a max face; ``acc`` is the [faces, 4] (E1, E2, H1, H2) accumulator array
    the library (GpuMesh.power_surfaces) or the oracle returns."""
    ptr = np.asarray(tables["ps_face_ptr"])
    codes = np.asarray(tables["ps_face_code"])
    dl = float(tables["dl"])
    out = np.zeros(len(ptr) - 1, dtype=np.complex128)
    for e in range(len(ptr) - 1):
        pwr = 0j
        for k in range(ptr[e], ptr[e + 1]):
            sign = 1.0 if codes[k] <= 3 else -1.0
            e1, e2, h1, h2 = acc[k]
            pwr = pwr + sign * (e1 * np.conj(h2) - e2 * np.conj(h1)) * dl * dl / 2.0
        out[e] = pwr
    return out


def power_surface_lines(freqs: Sequence[float], surface: Sequence[int], power: Sequence[complex]) -> List[str]:
    """The .frequency_domain_power_surface.fout file: its own header
    (``(A,I10)`` counts: the surfaces and the frequencies of the first one),
    then f, surface number, Re P, Im P, |Re P|, atan2(Im P, Re P), 10 log10 |Re P|."""
    n_surf = len(set(surface))
    n_freq = sum(1 for x in surface if x == surface[0]) if len(surface) else 0
    lines = [HEADER, "# Number of data points:" + f"{n_surf:10d}", "# Number of frequencies:" + f"{n_freq:10d}"]
    for f, num, p in zip(freqs, surface, power):
        p = complex(p)
        re = abs(p.real)
        db = 10.0 * math.log10(re) if re > 0.0 else -math.inf
        lines.append(fortran_e(f) + f"{int(num):5d}" +
                     "".join(fortran_e(x) for x in (p.real, p.imag, re, math.atan2(p.imag, p.real), db)))
    return lines


def oneport_calc(e1: complex, e2: complex, h1: complex, h2: complex,
                 d: float) -> Tuple[complex, complex, complex, complex]:
    """oneport_calc (POST_PROCESSOR/oneport.F90:206-249): from E and H at
    two output planes 2d apart in a uniform section, the propagation
    constant beta (real part made non-negative), the right- and left-going
    waves Er, El at the first plane and the wave impedance Z (real part made
    non-negative): the root P = exp(j beta d) of a P^2 + b P + c = 0 with
    a = c = E2 H1 + E1 H2, b = -2 (E1 H1 + E2 H2).  Returns (beta, Er, El, Z)."""
    a = e2 * h1 + e1 * h2
    b = -2.0 * (e1 * h1 + e2 * h2)
    c = e2 * h1 + e1 * h2
    s = cmath.sqrt(b * b - 4.0 * a * c)
    p1 = (-b + s) / (2.0 * a)
    beta = cmath.log(p1) / (2.0 * 1j * d)
    if beta.real < 0.0:
        beta = -beta
    p = cmath.exp(1j * beta * d)
    eit = (e2 * p - e1 * p * p * p) / (1.0 - p * p * p * p)
    z = (2.0 * eit * p - e1) / h1
    ert = -eit * p * p + e1 * p
    if z.real < 0.0:
        z = -z
    return beta, eit, ert, z


def oneport_lines(freqs: Sequence[float], ft: Sequence[Sequence[complex]], d_port: float,
                  l: float) -> Tuple[List[str], List[str]]:
    """Post-processor option 9, one-port analysis (POST_PROCESSOR/oneport.F90:35-205):
    ``ft`` holds E1, E2, H1, H2, the spectra on two planes ``d_port`` apart
    whose midpoint is ``l`` from the interface.  Returns the lines of the
    output file (per frequency, 11E14.5: f, beta, Z, the reflection
    coefficient R = (El/Er) exp(2 j beta l) with |R| and its dB, Re(w/beta),
    1 - |R|^2) and of its ``.Zs`` companion (f, the surface impedance
    Z (1+R)/(1-R) and its magnitude)."""
    E1, E2, H1, H2 = (np.asarray(x, dtype=np.complex128) for x in ft)
    d = d_port / 2.0
    out = ["    frequency       Re{Beta}     Im{Beta}       Re{Z}          Im{Z}"
           "         Re{R}          Im{R}        |R|          |R|(dB)      Re{w/Beta}    1-|R|**2"]
    zs_out = ["    frequency        Re{Zs}       Im{Zs}"]
    for k, f in enumerate(freqs):
        w = 2.0 * math.pi * f
        beta, ei, er, z = oneport_calc(E1[k], E2[k], H1[k], H2[k], d)
        r = (er / ei) * cmath.exp(2.0 * 1j * beta * l)
        zs = z * (1.0 + r) / (1.0 - r)
        vals = (f, beta.real, beta.imag, z.real, z.imag, r.real, r.imag, abs(r), 20.0 * math.log10(abs(r)),
                (w / beta).real, 1.0 - abs(r) ** 2)
        out.append("".join(fortran_e(v, 14, 5) for v in vals))
        zs_out.append("".join(fortran_e(v, 14, 5) for v in (f, zs.real, zs.imag, abs(zs))))
    return out, zs_out


def twoport_lines(freqs: Sequence[float], ft: Sequence[Sequence[complex]], d_port1: float, l1: float,
                  d_port2: float, l2: float, excitation_port: int = 1) -> List[str]:
    """Post-processor option 10, two-port analysis (POST_PROCESSOR/twoport.F90):
    ``ft`` holds the spectra E11, E12, H11, H12 (the two planes of port 1)
    and E21, E22, H21, H22 (port 2) on one frequency grid; each port's
    planes are ``d_port`` apart with their midpoint ``l`` from the interface.
    Returns the output file's lines: the list-directed title and per
    frequency (12E14.5) f, Re, Im, |.|, dB of S11 and S21 (S12 and S22 when
    port 2 is excited), then the reflected, transmitted and absorbed power."""
    E11, E12, H11, H12, E21, E22, H21, H22 = (np.asarray(x, dtype=np.complex128) for x in ft)
    if excitation_port == 1:
        title = " # f,dble(S11),dimag(S11),abs(S11),20.0*log10(abs(S11)),dble(S21),dimag(S21),abs(S21)," \
                "20.0*log10(abs(S21)), Pr, Pt, Pa"
    elif excitation_port == 2:
        title = " # f,dble(S12),dimag(S12),abs(S12),20.0*log10(abs(S12)),dble(S22),dimag(S22),abs(S22)," \
                "20.0*log10(abs(S22)), Pr, Pt, Pa"
    else:
        raise ValueError("excitation port must be 1 or 2")
    d1, d2 = d_port1 / 2.0, d_port2 / 2.0
    out = [title]
    for k, f in enumerate(freqs):
        beta1, er1, el1, _ = oneport_calc(E11[k], E12[k], H11[k], H12[k], d1)
        beta2, er2, el2, _ = oneport_calc(E22[k], E21[k], H22[k], H21[k], d2)
        if excitation_port == 1:
            sa = el1 * cmath.exp(1j * beta1 * l1) / (er1 * cmath.exp(-1j * beta1 * l1))  # S11
            sb = er2 * cmath.exp(1j * beta2 * l2) / (er1 * cmath.exp(-1j * beta1 * l1))  # S21
            pr, pt = abs(sa) ** 2, abs(sb) ** 2
        else:
            sa = el1 * cmath.exp(1j * beta1 * l1) / (el2 * cmath.exp(-1j * beta2 * l2))  # S12
            sb = er2 * cmath.exp(1j * beta2 * l2) / (el2 * cmath.exp(-1j * beta2 * l2))  # S22
            pr, pt = abs(sb) ** 2, abs(sa) ** 2
        vals = (f, sa.real, sa.imag, abs(sa), 20.0 * math.log10(abs(sa)), sb.real, sb.imag, abs(sb),
                20.0 * math.log10(abs(sb)), pr, pt, 1.0 - pr - pt)
        out.append("".join(fortran_e(v, 14, 5) for v in vals))
    return out


def transmission_cross_section_lines(power_rows: np.ndarray, field_rows: np.ndarray, field: str = "e") -> List[str]:
    """Post-processor option 15, transmission cross section
    (POST_PROCESSOR/transmission_cross_section.F90): from the transmitted
    power (|Re| of a power surface .fout, read_fout rows) and the cavity
    field's spectrum (|V| of an E or H .fout): TCS = Pt / Si with
    Si = 3 (|V|/sqrt 2)^2 scale / 2, scale 1/Z0 for E and Z0 for H.  The
    reference stores TCS through CMPLX() without a kind, so the value is
    rounded to single precision; the dB column is 10 log10 |TCS|."""
    fp, fe = power_rows[:, 0], field_rows[:, 0]
    if len(fp) != len(fe) or np.any(fp != fe):
        raise ValueError("the power and field files need the same frequencies")
    scale = 1.0 / Z0 if field.lower() == "e" else Z0
    lines = header(1, len(fp))
    # the power value is read through CMPLX() (single precision), the magnitude as printed
    for f, pw, mag in zip(fp, power_rows[:, 2].astype(np.float32).astype(np.float64), field_rows[:, 4]):
        e_rms = mag / math.sqrt(2.0)
        si = 3.0 * (e_rms ** 2) * scale / 2.0
        tcs = float(np.float32(abs(pw) / si))  # CMPLX(TCS): default (single) precision
        db = 10.0 * math.log10(abs(tcs)) if tcs != 0.0 else -math.inf
        lines.append(fortran_e(f) + f"{1:5d}" +
                     "".join(fortran_e(x) for x in (tcs, 0.0, abs(tcs), math.atan2(0.0, tcs), db)))
    return lines


def main(argv=None) -> int:
    """python -m ggi_tlm_b200.fout <file.tout> <point> <lin|log> <fmin> <fmax> <n_frequencies> <out.fout>:
    the post-processor's option 3 without its prompts."""
    import argparse

    from .tout import read_tout

    ap = argparse.ArgumentParser(prog="python -m ggi_tlm_b200.fout", description=main.__doc__.split("\n")[1].strip())
    ap.add_argument("tout")
    ap.add_argument("point", type=int)
    ap.add_argument("scale", choices=["lin", "log"])
    ap.add_argument("fmin", type=float)
    ap.add_argument("fmax", type=float)
    ap.add_argument("n_frequencies", type=int)
    ap.add_argument("out")
    a = ap.parse_args(argv)
    time, value = tout_series(read_tout(a.tout), a.point)
    if len(time) < 2:
        print(f"ERROR: output point {a.point} has fewer than two samples in {a.tout}")
        return 1
    freqs = frequencies(a.fmin, a.fmax, a.n_frequencies, a.scale)
    write_fout(a.out, freqs, fourier_transform(time, value, freqs))
    return 0


if __name__ == "__main__":
    import sys

    sys.exit(main())
