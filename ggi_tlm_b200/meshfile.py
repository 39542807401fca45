"""Reader for the reference's mesh files (NAME.mesh).

The reference's mesher writes the voxelised geometry once
(MESH/write_mesh.F90:95-305) and the solver reads it back
(MESH/read_mesh.F90:86-394) instead of voxelising the .inp geometry again.
The file is a sequence of Fortran list-directed records, one per line, each
possibly followed by a text label that the read ignores:

    dl
    nx ny nz
    mesh_xmin mesh_xmax            (and the y, z lines)
    n_volumes, then per volume: n_cells and n_cells lines  i j k point
    n_surfaces, then per surface: n_faces, its extent (3 lines), its cell
        range (3 lines) and n_faces lines  i j k point
    n_lines, then per line: n_segments and n_segments lines
        i1 j1 k1 point1 i2 j2 k2 point2
    n_points, then per point 3 lines: x y z / i j k / i j k point
    n_pml_volumes, then per PML volume: n_cells and n_cells lines  i j k point
    a label line, pml_volume_to_face(1:6)
    a label line, the PML thicknesses (xmin xmax / ymin ymax / zmin zmax)
    a label line, the PML reflection coefficients (three lines)
    a label line, the PML order

Cell indices are 1-based; ``point`` is a face code (face_xmin=1,
face_ymin=2, face_zmin=3, face_xmax=4, face_ymax=5, face_zmax=6) or the
cell centre (7), as TLM_MODULES/Mesh_Modules.F90:40-46 numbers them.
Files written before the PML section existed end after the points; they
read as meshes without PML volumes.

This is host-side input handling: the reader fills the geometry the GPU
path's tables are built from, so that meshes voxelised by the reference's own
mesher (spheres, triangulated surfaces) run without this package's
axis-aligned voxeliser.
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

FACE_XMIN, FACE_YMIN, FACE_ZMIN, FACE_XMAX, FACE_YMAX, FACE_ZMAX, CENTRE = 1, 2, 3, 4, 5, 6, 7
PML_FACE_NAMES = ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")  # pml_face_xmin=1 .. pml_face_zmax=6


@dataclass
class MeshSurface:
    """One surface of the mesh file: its extent in metres, its cell range
    and its faces as rows (i, j, k, face code)."""

    extent: Tuple[Tuple[float, float], Tuple[float, float], Tuple[float, float]]
    cell_range: Tuple[Tuple[int, int], Tuple[int, int], Tuple[int, int]]
    faces: np.ndarray


@dataclass
class MeshPoint:
    """One point of the mesh file: its coordinates, the cell that holds it
    and the cell face nearest to it (i, j, k, face code)."""

    xyz: Tuple[float, float, float]
    cell: Tuple[int, int, int]
    face: Tuple[int, int, int, int]


@dataclass
class MeshFile:
    dl: float
    n: Tuple[int, int, int]
    extent: Tuple[Tuple[float, float], Tuple[float, float], Tuple[float, float]]
    volumes: List[np.ndarray] = field(default_factory=list)        # per volume: rows (i, j, k, point)
    surfaces: List[MeshSurface] = field(default_factory=list)
    lines: List[np.ndarray] = field(default_factory=list)          # per line: rows of 8 (two segment points)
    points: List[MeshPoint] = field(default_factory=list)
    pml_volumes: List[np.ndarray] = field(default_factory=list)    # per PML volume: rows (i, j, k, point)
    pml_volume_to_face: Tuple[int, ...] = (0,) * 6
    pml_thickness: Tuple[float, ...] = (0.0,) * 6                  # metres: xmin, xmax, ymin, ymax, zmin, zmax
    pml_r: Tuple[float, ...] = (0.0,) * 6
    pml_order: Optional[int] = None
    has_pml_section: bool = False


_NUM = re.compile(r"^[+-]?(\d+\.?\d*|\.\d+)([eEdD][+-]?\d+)?$")


class _Records:
    """Fortran list-directed records: each read takes the first values of
    the next line and ignores the rest of it (the labels write_mesh adds)."""

    def __init__(self, lines: Sequence[str]):
        self.lines = [ln for ln in lines]
        self.pos = 0

    def done(self) -> bool:
        while self.pos < len(self.lines) and not self.lines[self.pos].strip():
            self.pos += 1
        return self.pos >= len(self.lines)

    def _next(self) -> str:
        if self.done():
            raise ValueError("mesh file ends early")
        ln = self.lines[self.pos]
        self.pos += 1
        return ln

    def values(self, n: int, kind=float) -> list:
        toks = [t for t in re.split(r"[\s,]+", self._next().strip()) if t]
        out = []
        for t in toks:
            if len(out) == n:
                break
            if not _NUM.match(t):
                raise ValueError(f"mesh file line {self.pos}: expected {n} numbers, found {t!r}")
            out.append(float(t.replace("d", "e").replace("D", "e")))
        if len(out) < n:
            raise ValueError(f"mesh file line {self.pos}: expected {n} numbers")
        if kind is int:
            if any(x != int(x) for x in out):
                raise ValueError(f"mesh file line {self.pos}: expected integers")
            return [int(x) for x in out]
        return out

    def label(self) -> None:
        self._next()

    def table(self, rows: int, cols: int) -> np.ndarray:
        a = np.zeros((rows, cols), dtype=np.int32)
        for r in range(rows):
            a[r] = self.values(cols, int)
        return a


def read_mesh(lines: Sequence[str]) -> MeshFile:
    """Parse the lines of a NAME.mesh file (read_mesh.F90:86-394)."""
    r = _Records(lines)
    dl = r.values(1)[0]
    n = tuple(r.values(3, int))
    ext = tuple(tuple(r.values(2)) for _ in range(3))
    m = MeshFile(dl=dl, n=n, extent=ext)
    for _ in range(r.values(1, int)[0]):                     # STAGE 1: volumes
        m.volumes.append(r.table(r.values(1, int)[0], 4))
    for _ in range(r.values(1, int)[0]):                     # STAGE 2: surfaces
        nf = r.values(1, int)[0]
        sext = tuple(tuple(r.values(2)) for _ in range(3))
        srng = tuple(tuple(r.values(2, int)) for _ in range(3))
        m.surfaces.append(MeshSurface(sext, srng, r.table(nf, 4)))
    for _ in range(r.values(1, int)[0]):                     # STAGE 3: lines (cable routes)
        m.lines.append(r.table(r.values(1, int)[0], 8))
    for _ in range(r.values(1, int)[0]):                     # STAGE 4: points
        xyz = tuple(r.values(3))
        cell = tuple(r.values(3, int))
        face = tuple(r.values(4, int))
        m.points.append(MeshPoint(xyz, cell, face))
    if r.done():  # a file written before the PML section existed
        return m
    m.has_pml_section = True
    for _ in range(r.values(1, int)[0]):                     # STAGE 5: PML volumes
        m.pml_volumes.append(r.table(r.values(1, int)[0], 4))
    r.label()
    m.pml_volume_to_face = tuple(r.values(6, int))
    r.label()
    m.pml_thickness = tuple(v for _ in range(3) for v in r.values(2))
    r.label()
    m.pml_r = tuple(v for _ in range(3) for v in r.values(2))
    r.label()
    m.pml_order = r.values(1, int)[0]
    return m


def check_cells(m: MeshFile, cells: np.ndarray, what: str) -> None:
    """Every row of ``cells`` is a cell centre (point 7) inside the mesh."""
    if cells.size == 0:
        return
    if np.any(cells[:, 3] != CENTRE):
        raise ValueError(f"{what}: a volume cell entry is not a cell centre (point 7)")
    for a in range(3):
        if cells[:, a].min() < 1 or cells[:, a].max() > m.n[a]:
            raise ValueError(f"{what}: a cell lies outside the {m.n[0]}x{m.n[1]}x{m.n[2]} mesh")


def connect_faces(m: MeshFile, faces: np.ndarray, what: str) -> List[Tuple[Tuple[int, int, int], int]]:
    """The faces of a surface as (cell on the + side of the face, axis):
    the min face of cell (i, j, k) along an axis is that cell's own min face,
    its max face is the min face of the next cell."""
    out = []
    for i, j, k, p in faces.tolist():
        if not 1 <= p <= 6:
            raise ValueError(f"{what}: face code {p} is not a face (1..6)")
        axis = (p - 1) % 3 + 1
        c = [i, j, k]
        if p > 3:
            c[axis - 1] += 1
        out.append(((c[0], c[1], c[2]), axis))
    return out


def pml_cells_from_mesh(m: MeshFile) -> Tuple[int, int, int, int, int, int]:
    """The PML depth in cells on each face, NINT(thickness/dl) as
    calc_pml_dist (TLM_PML_volume_materials.F90:465-466) takes it, after
    checking that the PML volumes' cells are exactly the box shell of those
    depths (the PML this package builds)."""
    t = tuple(int(np.rint(v / m.dl)) for v in m.pml_thickness)
    if not m.pml_volumes:
        return (0,) * 6
    nx, ny, nz = m.n
    got = np.zeros((nz, ny, nx), dtype=bool)
    for v in m.pml_volumes:
        check_cells(m, v, "PML volume")
        got[v[:, 2] - 1, v[:, 1] - 1, v[:, 0] - 1] = True
    z, y, x = np.meshgrid(np.arange(1, nz + 1), np.arange(1, ny + 1), np.arange(1, nx + 1), indexing="ij")
    want = ((x <= t[0]) | (x > nx - t[1]) | (y <= t[2]) | (y > ny - t[3]) | (z <= t[4]) | (z > nz - t[5]))
    if not np.array_equal(got, want):
        from .problem import UnsupportedFeature

        raise UnsupportedFeature("PML volumes that are not the box shell of the PML thicknesses")
    return t
