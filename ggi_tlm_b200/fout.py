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
