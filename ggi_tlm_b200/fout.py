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
20 log10 |V|.
"""
from __future__ import annotations

import math
from typing import List, Sequence, Tuple

import numpy as np

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
    read_frequency_domain_data takes them: from the printed Re and Im columns."""
    return rows[:, 0], rows[:, 2] + 1j * rows[:, 3]


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
