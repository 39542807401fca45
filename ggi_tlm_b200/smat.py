"""Reader for the reference's surface material files (``.smat``).

A dispersive thin layer is a two-port impedance matrix per polarisation
(TLM_MODULES/TLM_material_modules.F90: Z11_S..Z22_S(1:3)).  The file is read
as PROCESS_INPUT_FILE/read_surface_material_list.F90:150-290 reads it, with
Fortran list-directed input: a label line; fmin, fmax; then a comment line
and an S-filter (read_Sfilter, FILTER/filter_subroutines.F90:54-78: wnorm,
a order, a(0..order), b order, b(0..order)) for each of Z11, Z12, Z21, Z22 —
once for a DISPERSIVE layer (the same filters for the x, y and z
polarisations), three times (x, y, z) for an ANISOTROPIC_DISPERSIVE one.
"""
from __future__ import annotations

from typing import Sequence, Tuple

from .problem import SurfaceMaterial
from .vmat import _Records, _sfilter


def parse_smat(lines: Sequence[str], anisotropic: bool = False) -> Tuple[SurfaceMaterial, str, Tuple[float, float]]:
    """(material, label, (fmin, fmax)) of a .smat file's lines."""
    r = _Records(lines)
    label = r.line().strip().lower()
    fmin, fmax = r.values(2)
    pols = []
    for _ in range(3 if anisotropic else 1):
        z = []
        for _ in range(4):  # Z11, Z12, Z21, Z22
            r.line()  # comment
            z.append(_sfilter(r))
        pols.append(z)
    if not anisotropic:
        pols = [pols[0], list(pols[0]), list(pols[0])]
    return SurfaceMaterial(pols), label, (fmin, fmax)


def read_smat(path: str, anisotropic: bool = False) -> SurfaceMaterial:
    """The dispersive thin layer a .smat file describes."""
    with open(path) as f:
        return parse_smat(f.read().splitlines(), anisotropic)[0]
