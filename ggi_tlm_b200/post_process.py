"""The reference's post-processor (GGI_TLM_post_process) driven by its own
input file: ``python -m ggi_tlm_b200.post_process GGI_TLM_post_process_in.txt``
(or the lines on standard input), run in the directory that holds the
result files, as the reference's test cases run it.

The reference reads its answers to a sequence of prompts with Fortran
list-directed reads (a number takes the first field of its line, so the
test inputs' trailing remarks such as ``1e6 fmin`` are ignored).  Each
option here takes the same answers in the same order:

* 0 quit;
* 1 extract one output point's series from a time-domain file
  (extract_time_domain_data.F90): file, point, output file;
* 3 Fourier transform of one point of a time-domain file
  (fourier_transform.F90): file, point, lin|log, fmin, fmax, number of
  frequencies, output file;
* 6 combine two spectra, (A f1)/(B f2) + C (combine_frequency_domain_data.F90):
  file, point, file, point, A, B, C, output file;
* 9 one-port analysis (oneport.F90): four spectra (file, point) E1, E2, H1,
  H2, port separation, distance to the interface, output file (and its
  ``.Zs`` companion);
* 10 two-port analysis (twoport.F90): eight spectra, separation and
  distance of port 1 and of port 2, excitation port, output file;
* 13 extract a mode from a frequency output surface file (extract_mode.F90):
  file, then surface numbers each followed by its mode file, ended by 0;
* 15 transmission cross section (transmission_cross_section.F90): power
  spectrum, field spectrum, e|h, output file.

A spectrum is read as read_frequency_domain_data reads it: the rows of the
chosen point, values rounded to single precision.  Other options raise
``UnsupportedFeature``.
"""
from __future__ import annotations

import os
import sys
from typing import List, Optional, Sequence

import numpy as np

from . import fout, tout
from .problem import UnsupportedFeature


class _Answers:
    """The input file's lines, read as the prompts' list-directed reads."""

    def __init__(self, lines: Sequence[str]):
        self.lines = list(lines)
        self.pos = 0

    def line(self) -> str:
        while self.pos < len(self.lines) and not self.lines[self.pos].strip():
            self.pos += 1
        if self.pos >= len(self.lines):
            raise ValueError("post-processing input ends too early")
        ln = self.lines[self.pos]
        self.pos += 1
        return ln

    def more(self) -> bool:
        return any(x.strip() for x in self.lines[self.pos:])

    def name(self) -> str:  # read(*,'(A256)'): the line, trimmed
        return self.line().strip()

    def number(self) -> float:  # read(*,*): the first field
        return float(self.line().split()[0].replace("d", "e").replace("D", "E"))

    def integer(self) -> int:
        return int(self.line().split()[0])

    def word(self) -> str:
        return self.line().split()[0]


def _spectrum(a: _Answers, directory: str):
    path = os.path.join(directory, a.name())
    point = a.integer()
    rows = fout.read_fout(path)
    rows = rows[rows[:, 1] == point]
    if not len(rows):
        raise ValueError(f"{path}: no data for point {point}")
    return fout.spectrum(rows)


def read_frequency_output_surfaces(path: str) -> List[np.ndarray]:
    """The faces' data of each surface of a ``.frequency_output_surface.fout``
    as extract_mode.F90:120-196 reads it: per surface [faces] rows of cx, cy,
    cz and the phasor, the phasor held in single precision (``cmplx`` of
    default kind)."""
    with open(path) as f:
        lines = [ln for ln in f.read().splitlines()]
    pos = 1
    n_surfaces = int(lines[pos].split()[0]); pos += 1
    out = []
    for _ in range(n_surfaces):
        pos += 2
        n_points = int(lines[pos].split()[0]); pos += 2
        n_quads = int(lines[pos].split()[0]); pos += 2
        pos += 1 + n_points + n_quads  # frame count, corners, quads
        rows = np.loadtxt(lines[pos:pos + n_quads], ndmin=2)
        pos += n_quads
        out.append(rows)
    return out


def mode_lines(rows: np.ndarray) -> List[str]:
    """A mode file (extract_mode.F90:226-236, format(3I10,3E16.7)): cell,
    real and imaginary part and magnitude of each face's phasor, the parts
    rounded to single precision (``cmplx`` of default kind) and stored in a
    double complex (post_process_modules.F90:70), whose magnitude is taken
    in double precision."""
    z = rows[:, 3].astype(np.float32).astype(np.float64) + 1j * rows[:, 4].astype(np.float32).astype(np.float64)
    mag = np.abs(z)
    return ["".join(f"{int(c):10d}" for c in r[:3]) + tout.fortran_e(float(v.real), 16, 7) +
            tout.fortran_e(float(v.imag), 16, 7) + tout.fortran_e(float(m), 16, 7) for r, v, m in zip(rows, z, mag)]


def _write(path: str, lines: Sequence[str]) -> None:
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def run(lines: Sequence[str], directory: str = ".") -> List[str]:
    """Carry out every option of a post-processing input; returns the files written."""
    a = _Answers(lines)
    written: List[str] = []
    while a.more():
        option = a.integer()
        if option == 0:
            break
        if option in (1, 3):
            path = os.path.join(directory, a.name())
            point = a.integer()
            time, value = fout.tout_series(tout.read_tout(path), point)
            if option == 1:
                out = os.path.join(directory, a.name())
                _write(out, tout.header(1, len(time)) + [tout.data_line(t, 1, v, False) for t, v in zip(time, value)])
            else:
                scale = a.word().lower()
                fmin, fmax, n = a.number(), a.number(), a.integer()
                out = os.path.join(directory, a.name())
                freqs = fout.frequencies(fmin, fmax, n, scale)
                fout.write_fout(out, freqs, fout.fourier_transform(time, value, freqs))
            written.append(out)
        elif option == 6:
            (f1, v1), (f2, v2) = _spectrum(a, directory), _spectrum(a, directory)
            if len(f1) != len(f2) or np.any(f1 != f2):
                raise ValueError("combine: the two spectra need the same frequencies")
            A, B, C = a.number(), a.number(), a.number()
            out = os.path.join(directory, a.name())
            fout.write_fout(out, f1, fout.combine(v1, v2, A, B, C))
            written.append(out)
        elif option == 9:
            spec = [_spectrum(a, directory) for _ in range(4)]
            d_port, dist = a.number(), a.number()
            out = os.path.join(directory, a.name())
            lines9, zs = fout.oneport_lines(spec[0][0], [s[1] for s in spec], d_port, dist)
            _write(out, lines9)
            _write(out + ".Zs", zs)
            written += [out, out + ".Zs"]
        elif option == 10:
            spec = [_spectrum(a, directory) for _ in range(8)]
            d1, l1, d2, l2 = a.number(), a.number(), a.number(), a.number()
            port = a.integer()
            out = os.path.join(directory, a.name())
            _write(out, fout.twoport_lines(spec[0][0], [s[1] for s in spec], d1, l1, d2, l2, port))
            written.append(out)
        elif option == 13:
            surfaces = read_frequency_output_surfaces(os.path.join(directory, a.name()))
            while True:
                k = a.integer()
                if k == 0:
                    break
                if not 1 <= k <= len(surfaces):
                    raise ValueError(f"extract mode: surface {k} is not between 1 and {len(surfaces)}")
                out = os.path.join(directory, a.name())
                _write(out, mode_lines(surfaces[k - 1]))
                written.append(out)
        elif option == 15:
            power_path, power_point = os.path.join(directory, a.name()), a.integer()
            field_path, field_point = os.path.join(directory, a.name()), a.integer()
            kind = a.word()
            out = os.path.join(directory, a.name())
            pw, fd = fout.read_fout(power_path), fout.read_fout(field_path)
            _write(out, fout.transmission_cross_section_lines(pw[pw[:, 1] == power_point],
                                                              fd[fd[:, 1] == field_point], kind))
            written.append(out)
        else:
            raise UnsupportedFeature(f"post-processing option {option}")
    return written


def main(argv: Optional[Sequence[str]] = None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    if argv:
        with open(argv[0]) as f:
            lines = f.read().splitlines()
    else:
        lines = sys.stdin.read().splitlines()
    for path in run(lines, "."):
        print("wrote", path)
    return 0


if __name__ == "__main__":
    sys.exit(main())
