"""Reader for the reference's volume material files (``.vmat``).

The file is read as PROCESS_INPUT_FILE/read_volume_material_list.F90:128-156
reads it, with Fortran list-directed input: a label line; fmin, fmax; a
comment line; the permittivity S-filter (read_Sfilter,
FILTER/filter_subroutines.F90:54-78: wnorm, a order, a(0..order), b order,
b(0..order)); sigma_e; a comment line; the permeability S-filter; sigma_m.
A list-directed read takes the values it needs from one or more lines and
discards the rest of its last line, so trailing ``# ...`` remarks are
ignored.  The result is a dispersive VolumeMaterial for the problem tables.
"""
from __future__ import annotations

import re
from typing import Iterator, List, Sequence, Tuple

from .problem import MAT_DISPERSIVE, Sfilter, VolumeMaterial

_SEP = re.compile(r"[\s,]+")


class _Records:
    """Fortran-style sequential records: whole lines, or N values from one or more lines."""

    def __init__(self, lines: Sequence[str]):
        self._it: Iterator[str] = iter(lines)

    def line(self) -> str:
        try:
            return next(self._it)
        except StopIteration:
            raise ValueError("volume material file ends too early") from None

    def values(self, n: int) -> List[float]:
        out: List[float] = []
        while len(out) < n:
            for tok in _SEP.split(self.line().strip()):
                if not tok:
                    continue
                try:
                    out.append(float(tok.replace("d", "e").replace("D", "e")))
                except ValueError:
                    break  # a remark ends the values on this line
                if len(out) == n:
                    break
        return out


def _sfilter(r: _Records) -> Sfilter:
    wnorm = r.values(1)[0]
    na = int(r.values(1)[0])
    a = r.values(na + 1)
    nb = int(r.values(1)[0])
    b = r.values(nb + 1)
    return Sfilter(wnorm, a, b)


def parse_vmat(lines: Sequence[str]) -> Tuple[VolumeMaterial, str, Tuple[float, float]]:
    """(material, label, (fmin, fmax)) of a .vmat file's lines."""
    r = _Records(lines)
    label = r.line().strip().lower()
    fmin, fmax = r.values(2)
    r.line()  # comment
    eps = _sfilter(r)
    sigma_e = r.values(1)[0]
    r.line()  # comment
    mu = _sfilter(r)
    sigma_m = r.values(1)[0]
    return VolumeMaterial(MAT_DISPERSIVE, eps, sigma_e, mu, sigma_m), label, (fmin, fmax)


def read_vmat(path: str) -> VolumeMaterial:
    """The dispersive volume material a .vmat file describes."""
    with open(path) as f:
        return parse_vmat(f.read().splitlines())[0]
