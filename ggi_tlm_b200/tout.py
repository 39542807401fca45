"""Time-domain output files in the reference's text format.

GGI_TLM writes its time-domain results (``.field.tout`` and friends) as a
three-line header (write_time_domain_header_data,
FILE_HANDLING/read_write_header_data.F90:30-50) followed by one line per
output point and output step in the Fortran format ``(E16.7,I5,E16.7)``
(time_domain_output_format, TLM_MODULES/File_information.F90:235): the
time, the 1-based output point number and the value, with values below
1e-30 in magnitude written as 0 (output_points.F90:586-600).  This module
writes the same bytes from the series the library returns, so the files the
reference's post-processing reads are unchanged.
"""
from __future__ import annotations

from typing import Iterable, List, Optional, Sequence, Tuple

import math

import numpy as np

HEADER = "# Time Domain Data"  # time_domain_output_file_header, File_information.F90:263


def fortran_e(value: float, width: int = 16, digits: int = 7) -> str:
    """Fortran ``Ew.d`` editing as gfortran writes it: ``0.ddddddd`` with
    the exponent as ``E+xx`` (or ``+xxx`` without the E when it needs three
    digits), right-justified in ``width`` columns."""
    v = float(value)
    if v != v:
        return "NaN".rjust(width)
    if v in (float("inf"), float("-inf")):  # gfortran writes the word, signed only when negative
        return ("-Infinity" if v < 0 else "Infinity").rjust(width)
    if v == 0.0:  # a negative zero keeps its sign, as gfortran writes it
        body = "0." + "0" * digits + "E+00"
        return (("-" if math.copysign(1.0, v) < 0 else "") + body).rjust(width)
    s = f"{abs(v):.{digits - 1}e}"  # d.dddddde+xx, correctly rounded to `digits` significant digits
    mant, exp = s.split("e")
    e = int(exp) + 1
    body = "0." + mant.replace(".", "")
    body += (f"E{'+' if e >= 0 else '-'}{abs(e):02d}" if abs(e) < 100 else f"{'+' if e >= 0 else '-'}{abs(e):03d}")
    return (("-" if v < 0 else "") + body).rjust(width)


def header(n_points: int, n_timesteps: int) -> List[str]:
    """The three header lines: the title, then ``(A25,I10)`` counts."""
    return [HEADER, "# Number of data points: " + f"{n_points:10d}", "# Number of Timesteps  : " + f"{n_timesteps:10d}"]


def data_line(time: float, point: int, value: float, flush_small: bool = True) -> str:
    """One ``(E16.7,I5,E16.7)`` line; with ``flush_small`` (the output files)
    |value| < 1e-30 is written as 0, without it (the excitation file) as is."""
    v = 0.0 if flush_small and abs(value) < 1e-30 else float(value)
    return fortran_e(time) + f"{int(point):5d}" + fortran_e(v)


def write_tout(path: str, rows: Iterable[Tuple[float, int, float]], n_points: int, n_timesteps: int) -> None:
    """Write a .tout file from (time, point number, value) rows in file order."""
    with open(path, "w") as f:
        for line in header(n_points, n_timesteps):
            f.write(line + "\n")
        for t, p, v in rows:
            f.write(data_line(t, p, v) + "\n")


def output_flag(timestep: int, timing: Optional[Tuple[int, int, int]]) -> bool:
    """get_output_flag (OUTPUT/output.F90:570-600): output on the steps
    first..last that are a multiple of interval after first; None (no
    timing block) is every step."""
    if timing is None:
        return True
    first, last, interval = timing
    return first <= timestep <= last and (timestep - first) % interval == 0


def field_rows(tables: dict, centre: np.ndarray, face: np.ndarray, first_step: int = 1,
               timing: Optional[Sequence[Optional[Tuple[int, int, int]]]] = None) -> List[Tuple[float, int, float]]:
    """Rows of a .field.tout for output points sampled every step, in the
    reference's order: each step the cell-centre points at the cell-output
    time (timestep-1)*dt (cell_output_point, output_points.F90:586-600),
    then the face points half a step later (face_output_points, :428-441).
    ``centre`` is [n_centre_points, steps] (probe_series), ``face`` is
    [n_face_points, steps] (GpuMesh.face_output); the point numbers are the
    tables' ``out_point_no`` / ``fprobe_point_no``.  ``timing``, indexed by
    output point number - 1, gives each point's (first, last, interval)
    output steps or None for every step (the .inp reader's output_timing)."""
    dt = float(tables["dt"])
    cno = np.asarray(tables.get("out_point_no", np.arange(1, centre.shape[0] + 1)))
    fno = np.asarray(tables.get("fprobe_point_no", np.arange(1, face.shape[0] + 1)))
    n_steps = centre.shape[1] if centre.size else (face.shape[1] if face.size else 0)

    def on(point: int, timestep: int) -> bool:
        return timing is None or output_flag(timestep, timing[point - 1])

    rows = []
    for s in range(n_steps):
        timestep = first_step + s
        time = (timestep - 1) * dt
        for k in range(centre.shape[0]):
            if on(int(cno[k]), timestep):
                rows.append((time, int(cno[k]), float(centre[k, s])))
        time = time + dt / 2.0
        for k in range(face.shape[0]):
            if on(int(fno[k]), timestep):
                rows.append((time, int(fno[k]), float(face[k, s])))
    return rows


def excitation_rows(tables: dict) -> List[Tuple[float, int, float]]:
    """Rows of the .excitation.tout file initialise_excitation_functions writes
    (EXCITATION/excitation.F90:186-553): for each function in turn, its value
    at every timestep at time (timestep-1)*dt, without the small-value flush."""
    dt = float(tables["dt"])
    val = np.asarray(tables["fn_value"]).reshape(int(tables["n_functions"]), -1)
    return [((ts - 1) * dt, e + 1, float(val[e, ts - 1])) for e in range(val.shape[0])
            for ts in range(1, val.shape[1] + 1)]


def read_tout(path: str) -> np.ndarray:
    """(time, point, value) rows of a .tout file as an [n, 3] array."""
    return np.loadtxt(path, comments="#", ndmin=2)


def format_rows(rows: Sequence[Tuple[float, int, float]]) -> List[str]:
    return [data_line(t, p, v) for t, p, v in rows]
