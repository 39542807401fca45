"""Reader for the reference's problem input files (``.inp``).

A GGI_TLM input is a sequence of packets: a keyword line (the names read by
PROCESS_INPUT_FILE/read_input_file_geometry.F90 and read_input_file_solver.F90)
followed by its data, read with Fortran list-directed input (values taken
from as many lines as needed, the rest of the last line ignored, reals such
as ``3.0-3`` allowed).  ``read_inp`` turns the packets the time loop needs
into a ProblemSpec, restating the reference's set-up for axis-aligned
geometry without rotations:

- the mesh (set_mesh_parameters.F90:55-100): ``Mesh_cell_dimension`` gives
  nx = NINT(extent / dl); ``Mesh_dimensions_in_cells`` gives dl as the mean
  of the three spacings (evaluated as the reference's build does, see
  cases.cubic_mesh_dl);
- points, volumes and surfaces with a transformation of zero Euler angles
  (GEOMETRY/transformations.F90: the point plus the translation);
  ``rectangular_block`` volumes take the cells whose centres lie inside,
  ``rectangle`` / ``xplane`` / ``yplane`` / ``zplane`` surfaces on a cell
  boundary become face patches, ``rectangular_block`` surfaces closed boxes;
- PML thicknesses in metres, NINT(t / dl) cells (TLM_PML_volume_materials.F90:465);
- volume materials from ``.vmat`` files (ggi_tlm_b200.vmat), excitation
  functions, point excitations, the Huygens surface, output points,
  ``Simulation_time`` (n_timesteps = NINT(T / dt)) and ``set_small_to_zero``.

Packets that only post-processing or other programs use are listed in
``InpProblem.skipped``; geometry or packets that the GPU path does not
support raise UnsupportedFeature.
"""
from __future__ import annotations

import os
import re
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

from .meshfile import MeshFile, check_cells, connect_faces, pml_cells_from_mesh, read_mesh
from .problem import (C0, MAT_PEC, MAT_PMC, SOURCE_HARD, SOURCE_SOFT, Block, CellList, DFTSurface, ExcitationFunction,
                      FarFieldSurface, FrequencyOutputVolume, HuygensBox, HuygensOuter, HuygensPlane, ModeOutput,
                      OutputPoint,
                      OutputSurface, OutputVolume, PointExcitation, PowerSurface, ProblemSpec, RCSSurface, SARVolume,
                      SurfaceMaterial, SurfaceSheet, UnsupportedFeature, VolumeMaterial, Z0, _region_mask, nint)

GEOMETRY_PACKETS = ["periodic_boundary", "mesh_outer_boundary_dimension", "mesh_dimensions_in_cells",
                    "mesh_cell_dimension", "volume_list", "surface_list", "line_list", "point_list", "pml",
                    "new_mesh_generation", "no_geometry_vtk_files"]
SOLVER_PACKETS = ["simulation_time", "volume_material_list", "surface_material_list",
                  "outer_boundary_reflection_coefficient", "excitation_function_list", "excitation_point_list",
                  "excitation_surface_list", "excitation_volume_list", "huygens_surface", "output_point_list",
                  "ngspice_node_output_list", "output_surface_list", "output_volume_list",
                  "output_volume_average_list", "output_volume_peak_list", "sar_volume_list",
                  "far_field_surface_list", "periodic_boundary_far_field_surface", "frequency_output_surface_list",
                  "frequency_output_volume_list_xyz", "frequency_output_volume_list",
                  "frequency_domain_power_surface_list", "rcs_surface", "excitation_mode_list", "output_mode_list",
                  "mode_stir_surface_list", "bicubic_warp_flag", "frequency_scale_flag", "compress_output_files",
                  "reduced_c_factor", "wrapping_boundary_conditions", "random_number_seed",
                  "ngspice_timestep_factor", "ngspice_lpf_alpha", "set_small_to_zero"]
# read_input_file_cables.F90: the cable model's packets, in the same file
CABLE_PACKETS = ["cable_geometry_list", "cable_list", "cable_junction_list", "cable_output_list",
                 "tlm_cell_equivalent_radius_factor", "capacitance_equivalent_radius_factor",
                 "inductance_equivalent_radius_factor", "lc_correction_type_geometry_scale",
                 "lc_correction_type_subtract_cell_inductance", "max_cable_bundle_diameter_factor"]
PACKETS = set(GEOMETRY_PACKETS + SOLVER_PACKETS + CABLE_PACKETS)
# packets that change nothing the time loop computes here: mesh and output
# file options, lines (used by cables only), the random seed (used by the
# random options, which are refused) and the cable model's factors
NEUTRAL = {"new_mesh_generation", "no_geometry_vtk_files", "compress_output_files", "line_list",
           "random_number_seed", "tlm_cell_equivalent_radius_factor", "capacitance_equivalent_radius_factor",
           "inductance_equivalent_radius_factor", "lc_correction_type_geometry_scale",
           "lc_correction_type_subtract_cell_inductance", "max_cable_bundle_diameter_factor"}
# packets of other parts of the reference the GPU path does not run
UNSUPPORTED = {"periodic_boundary",
               "ngspice_node_output_list", "periodic_boundary_far_field_surface",
               "mode_stir_surface_list", "ngspice_timestep_factor",
               "ngspice_lpf_alpha", "cable_geometry_list", "cable_list", "cable_junction_list", "cable_output_list"}
# run by the GPU path but not read here
NOT_READ = set()
# packets read_inp turns into the spec
HANDLED = {"wrapping_boundary_conditions", "mesh_outer_boundary_dimension", "mesh_cell_dimension", "mesh_dimensions_in_cells", "pml",
           "volume_list", "surface_list", "point_list", "simulation_time", "volume_material_list",
           "surface_material_list", "outer_boundary_reflection_coefficient", "excitation_function_list",
           "excitation_point_list", "excitation_surface_list", "excitation_volume_list", "excitation_mode_list",
           "huygens_surface", "output_point_list", "output_surface_list", "output_mode_list",
           "output_volume_list", "output_volume_average_list", "output_volume_peak_list",
           "frequency_output_volume_list", "frequency_output_volume_list_xyz", "frequency_output_surface_list",
           "far_field_surface_list", "rcs_surface", "frequency_domain_power_surface_list", "sar_volume_list",
           "set_small_to_zero", "reduced_c_factor", "bicubic_warp_flag", "frequency_scale_flag"}

# field component names (TLM_MODULES/TLM_Modules.F90:149-161): read_field_component
# takes Ex..Hz, read_field_or_currrent_component also Jx..Jz, both comparing
# the whole line; read_field_component_surface_output compares the first two
# columns only ('(A2)') and adds the magnitudes em, hm, jm
_FIELD = {"ex": "Ex", "ey": "Ey", "ez": "Ez", "hx": "Hx", "hy": "Hy", "hz": "Hz"}
_FIELD_OR_CURRENT = {**_FIELD, "jx": "Jx", "jy": "Jy", "jz": "Jz"}
_SURFACE_FIELD = {**_FIELD_OR_CURRENT, "em": "Em", "hm": "Hm", "jm": "Jm"}
_FACES = {"centre", "xmin", "xmax", "ymin", "ymax", "zmin", "zmax"}  # read_centre_or_face
_FACE_OF_CODE = {1: "xmin", 2: "ymin", 3: "zmin", 4: "xmax", 5: "ymax", 6: "zmax"}  # Mesh_Modules.F90:40-46
# parameters per geometry type (read_volume_list.F90:107-159, read_surface_list.F90:108-220);
# the types marked with a file name read that line before the parameters
_VOLUME_PARAMS = {"rectangular_block2": 6, "rectangular_block": 3, "cylinder": 2, "sphere": 1, "tet": 12, "hex": 24,
                  "pyramid_ram": 3, "pyramid": 2, "tet_volume_mesh": 1, "fill_surface": 1}
_SURFACE_PARAMS = {"rectangular_block2": 6, "rectangular_block": 3, "cylinder": 2, "sphere": 1, "hemisphere": 1,
                   "rectangle": 2, "circle": 1, "quad": 12, "xplane": 6, "yplane": 6, "zplane": 6, "triangle": 9,
                   "annulus": 2, "split_ring": 3, "helix": 6, "triangulated_surface": 2,
                   "vtk_triangulated_surface": 2, "stl_triangulated_surface": 2}
_WITH_FILE = {"tet_volume_mesh", "triangulated_surface", "vtk_triangulated_surface", "stl_triangulated_surface"}
# parameters per excitation function type, read_excitation_function_list.F90:108-160
_N_PARAMS = {"impulse": 1, "gaussian_step": 3, "step": 2, "gaussian": 3, "sinusoid": 3, "gaussian_sinusoid": 5,
             "gaussian_step_sinusoid": 5, "double_exponential": 3, "differential_gaussian": 3,
             "sinusoidal_pulse": 7, "ring_wave": 4}
# noise draws from the Fortran run-time's random number generator, which the tables cannot reproduce
_OTHER_FUNCTIONS = {"noise"}

_REAL = re.compile(r"^([+-]?(?:\d+\.?\d*|\.\d+))(?:[eEdD]([+-]?\d+)|([+-]\d+))?$")


def fortran_real(tok: str) -> float:
    """A real as Fortran list-directed input reads it, exponent letter optional
    (``1.0e-3``, ``1.0d-3``, ``1.0-3``)."""
    m = _REAL.match(tok)
    if not m:
        raise ValueError(tok)
    exp = m.group(2) or m.group(3)
    return float(m.group(1) + ("e" + exp if exp else ""))


class Records:
    """The data lines of one packet, read as Fortran sequential records."""

    def __init__(self, name: str, lines: Sequence[str]):
        self.name = name
        self.lines = list(lines)
        self.pos = 0

    def line(self) -> str:
        if self.pos >= len(self.lines):
            raise ValueError(f"{self.name} packet ends too early")
        self.pos += 1
        return self.lines[self.pos - 1]

    def text(self) -> str:
        """The next line read with '(A)' and converted to lower case; the
        reference compares it whole with a keyword (trailing blanks ignored)."""
        return self.line().rstrip().lower()

    def peek_text(self, width: int = 256) -> str:
        """The next line's first ``width`` columns in lower case, without
        consuming it (a read followed by BACKSPACE)."""
        if self.pos >= len(self.lines):
            return ""
        return self.lines[self.pos][:width].rstrip().lower()

    def values(self, n: int) -> List[float]:
        """``n`` values of a list-directed read: as many lines as needed, the
        rest of the last line ignored (the remarks after the numbers), a
        value written ``r*c`` repeated r times; any other text where a value
        is still needed is a read error, as in the reference."""
        out: List[float] = []
        while len(out) < n:
            line = self.line()
            for tok in re.split(r"[\s,]+", line.strip()):
                if not tok:
                    continue
                rep = re.match(r"^(\d+)\*(.+)$", tok)
                try:
                    vals = [fortran_real(rep.group(2))] * int(rep.group(1)) if rep else [fortran_real(tok)]
                except ValueError:
                    raise ValueError(f"{self.name} packet: expected a number, read {line.strip()!r}") from None
                out.extend(vals)
                if len(out) >= n:
                    break
        return out[:n]

    def ints(self, n: int) -> List[int]:
        return [int(v) for v in self.values(n)]


def split_packets(lines: Sequence[str]) -> List[Tuple[str, List[str]]]:
    """(keyword, data lines) of each packet in file order; blank lines and
    lines before the first keyword (the title) are dropped."""
    out: List[Tuple[str, List[str]]] = []
    for raw in lines:
        line = raw.rstrip("\n")
        if not line.strip():
            continue
        tok = line.split()
        if tok[0].lower() in PACKETS and (len(tok) == 1 or tok[1][0] in "!#"):
            out.append((tok[0].lower(), []))
        elif out:
            out[-1][1].append(line)
    return out


@dataclass
class Mesh:
    xmin: float
    ymin: float
    zmin: float
    dl: float
    n: Tuple[int, int, int]

    def lo(self, axis: int) -> float:
        return (self.xmin, self.ymin, self.zmin)[axis]

    def cell_of(self, p: Sequence[float]) -> Tuple[int, int, int]:
        """get_cell_number: int((p - min) * (1/dl)) + 1 per axis, the
        multiplication by 1/dl as the reference's build evaluates it."""
        return tuple(int((p[a] - self.lo(a)) * (1.0 / self.dl)) + 1 for a in range(3))

    def centres_in(self, axis: int, lo: float, hi: float) -> Tuple[int, int]:
        """1-based range of cells along ``axis`` whose centres lie in [lo, hi];
        a centre on the boundary is ambiguous under rounding and is refused."""
        cells = []
        for c in range(1, self.n[axis] + 1):
            x = self.lo(axis) + (c - 0.5) * self.dl
            if min(abs(x - lo), abs(x - hi)) < 1e-9 * self.dl:
                raise UnsupportedFeature("a cell centre lies on a volume or surface boundary")
            if lo < x < hi:
                cells.append(c)
        if not cells:
            raise UnsupportedFeature("a volume or surface contains no cell")
        return cells[0], cells[-1]

    def boundary(self, axis: int, x: float) -> int:
        """The cell boundary index k (between cells k and k+1) at coordinate x."""
        k = (x - self.lo(axis)) / self.dl
        if abs(k - round(k)) > 1e-6:
            raise UnsupportedFeature("a surface does not lie on cell boundaries")
        return int(round(k))


def _transform(r: Records, what: str) -> Tuple[float, float, float]:
    """A transformation (3 Euler angles in degrees, 3 translations); only zero angles are supported."""
    t = r.values(6)
    if any(v != 0.0 for v in t[:3]):
        raise UnsupportedFeature(f"rotated {what}: only zero Euler angles are supported")
    return t[3], t[4], t[5]


@dataclass
class InpProblem:
    """The spec, the packets read but without effect on the time loop
    (``skipped``), each output point's output steps, and the parameters only
    the host-side post-processing uses (``post``: "far_field" -> one dict of
    angle ranges per far-field surface, "rcs" -> the frequency range,
    "sar_density" -> one density per SAR volume)."""

    spec: ProblemSpec
    skipped: List[str] = field(default_factory=list)
    # per output point: (first, last, interval) timesteps, or None for every step
    output_timing: List[Optional[Tuple[int, int, int]]] = field(default_factory=list)
    post: Dict[str, object] = field(default_factory=dict)




@dataclass
class Shape:
    """A volume or surface of the geometry lists after its transformation:
    ``kind`` is the reference's type name, ``par`` its parameters and ``tr``
    the translation (None for types this reader does not voxelise), and
    ``rough`` marks a surface with a surface_roughness line."""

    kind: str
    par: Optional[List[float]]
    tr: Optional[Tuple[float, float, float]]
    rough: bool = False
    rotated: bool = False


def _geometry_list(r: Records, what: str, counts: Dict[str, int], supported: set) -> Dict[int, Shape]:
    """read_volume_list / read_surface_list: number, type line, [file name],
    parameters, [surface_roughness + values], transformation."""
    out: Dict[int, Shape] = {}
    n = r.ints(1)[0]
    for k in range(1, n + 1):
        if r.ints(1)[0] != k:
            raise ValueError(f"{r.name} packet: {what}s must be numbered in order")
        kind = r.text()
        if kind not in counts:
            raise ValueError(f"{r.name} packet: unknown {what} type {kind!r}")
        if kind in _WITH_FILE:
            r.line()
        par = r.values(counts[kind])
        rough = False
        if what == "surface" and r.peek_text(17) == "surface_roughness":
            r.line()
            r.values(1 if kind == "sphere" else 2)
            rough = True
        t = r.values(6)  # the transformation: three Euler angles, three translations
        if kind in supported and not any(v != 0.0 for v in t[:3]):
            out[k] = Shape(kind, par, (t[3], t[4], t[5]), rough)
        else:  # refused when something uses it
            out[k] = Shape(kind, None, None, rough, rotated=kind in supported)
    return out


def _block_cells(mesh: Mesh, par, tr, kind: str = "rectangular_block") -> Block:
    """The cells whose centres lie inside an axis-aligned block: of sides
    ``par`` centred on the translation ``tr`` (build_volume_rectangular_block.F90),
    or for rectangular_block2 between the corners par[0:3] and par[3:6], each
    pair sorted, moved by ``tr`` (build_volume_rectangular_block2.F90)."""
    if kind == "rectangular_block2":
        lo = [min(par[a], par[3 + a]) + tr[a] for a in range(3)]
        hi = [max(par[a], par[3 + a]) + tr[a] for a in range(3)]
    else:
        lo = [tr[a] - par[a] / 2.0 for a in range(3)]
        hi = [tr[a] + par[a] / 2.0 for a in range(3)]
    rng = [mesh.centres_in(a, lo[a], hi[a]) for a in range(3)]
    return Block(rng[0][0], rng[0][1], rng[1][0], rng[1][1], rng[2][0], rng[2][1])


def _surface_cells(mesh: Mesh, s: Shape, what: str):
    """("box", ((i0, i1), (j0, j1), (k0, k1))) for a rectangular_block surface,
    or ("plane", (axis, index, r0, r1), orient) for a planar one.  ``orient``
    is +1 when the triangles' normal (v3-v1)x(v2-v1) points along -axis, the
    orientation of build_surface_rectangle.F90 that HuygensPlane side 1
    describes, and -1 when it points along +axis: build_surface_xplane.F90
    (and y/z) order the corners so that the normal is +x for y2>y1, z2>z1,
    -y for x2>x1, z2>z1 and +z for x2>x1, y2>y1."""
    if s.rotated:
        raise UnsupportedFeature(f"{what} on a rotated {s.kind}: only zero Euler angles are supported")
    if s.par is None:
        raise UnsupportedFeature(f"{what} on a surface of type {s.kind!r}")
    if s.rough:
        raise UnsupportedFeature(f"{what} on a surface with random roughness")
    par, tr = s.par, s.tr
    if s.kind in ("rectangular_block", "rectangular_block2"):
        # both builders give every triangle an inward normal (the HuygensBox convention)
        b = _block_cells(mesh, par, tr, s.kind)
        return "box", ((b.i0, b.i1), (b.j0, b.j1), (b.k0, b.k1)), 1
    if s.kind == "rectangle":  # lx by ly in the local xy-plane, centred on the translation
        axis, orient = 2, 1
        lo = [tr[0] - par[0] / 2.0, tr[1] - par[1] / 2.0, tr[2]]
        hi = [tr[0] + par[0] / 2.0, tr[1] + par[1] / 2.0, tr[2]]
    else:
        axis = {"xplane": 0, "yplane": 1, "zplane": 2}[s.kind]
        p1 = [par[a] + tr[a] for a in range(3)]
        p2 = [par[3 + a] + tr[a] for a in range(3)]
        if p1[axis] != p2[axis]:
            raise ValueError(f"{s.kind} surface: the two corners differ in the normal coordinate")
        d = [p2[a] - p1[a] for a in range(3)]
        normal = (d[1] * d[2], -(d[0] * d[2]), d[0] * d[1])[axis]
        if normal == 0.0:
            raise UnsupportedFeature(f"{s.kind} surface of zero area")
        orient = -1 if normal > 0.0 else 1
        lo, hi = [min(a, b) for a, b in zip(p1, p2)], [max(a, b) for a, b in zip(p1, p2)]
    t = [a for a in range(3) if a != axis]
    return "plane", (axis + 1, mesh.boundary(axis, lo[axis]), mesh.centres_in(t[0], lo[t[0]], hi[t[0]]),
                     mesh.centres_in(t[1], lo[t[1]], hi[t[1]])), orient


def _timing(r: Records, dt: float) -> Optional[Tuple[int, int, int]]:
    """read_output_time_information.F90 followed by set_output_time_information
    (OUTPUT/output.F90:487-545): an optional output_timestep_information
    (three integers) or output_time_information (three times, NINT(t/dt))
    block, each value raised to at least 1; None when the block is absent
    (every step)."""
    w = r.peek_text()
    if w == "output_timestep_information":
        r.line()
        first, last, step = (r.ints(1)[0] for _ in range(3))
    elif w == "output_time_information":
        r.line()
        first, last, step = (nint(r.values(1)[0] / dt) for _ in range(3))
    else:
        return None
    return max(first, 1), max(last, 1), max(step, 1)


def _steps(t: Optional[Tuple[int, int, int]]) -> dict:
    if t is None:
        return dict(first_step=1, last_step=None, interval=1)
    return dict(first_step=t[0], last_step=t[1], interval=t[2])


def _component(r: Records, names: Dict[str, str], width: int = 256) -> str:
    key = r.line()[:width].rstrip().lower()
    if key not in names:
        raise ValueError(f"{r.name} packet: unknown field component {key!r}")
    return names[key]


def _face(r: Records) -> str:
    f = r.text()
    if f not in _FACES:
        raise ValueError(f"{r.name} packet: expected centre or a face name, got {f!r}")
    return f


def _logical(tok: str) -> bool:
    """A list-directed LOGICAL value: optional '.', then T or F."""
    t = tok.strip().lower().lstrip(".")
    if not t or t[0] not in "tf":
        raise ValueError(f"not a logical value: {tok!r}")
    return t[0] == "t"


def _samples(lines: Sequence[str], n_ignore: int, n_time: int, n_value: int) -> Tuple[List[float], List[float]]:
    """read_excitation_function_list.F90:182-215: skip n_ignore lines, then
    list-directed records of max(n_time, n_value) values to the end of the
    file, keeping the n_time-th as the time and the n_value-th as the value."""
    r = Records("excitation function file", list(lines)[n_ignore:])
    n = max(n_time, n_value)
    times: List[float] = []
    values: List[float] = []
    while any(x.strip() for x in r.lines[r.pos:]):
        try:
            rec = r.values(n)
        except ValueError as e:
            if "ends too early" in str(e):
                break  # the end of the file inside a record ends the samples
            raise
        times.append(rec[n_time - 1])
        values.append(rec[n_value - 1])
    if not times:
        raise ValueError("an excitation function file without samples")
    return times, values


def read_inp(lines: Sequence[str], material: Callable[[str], VolumeMaterial],
             open_file: Optional[Callable[[str], Sequence[str]]] = None,
             mesh_file: Optional[MeshFile] = None,
             thin_layer: Optional[Callable[[str, bool], SurfaceMaterial]] = None) -> InpProblem:
    """The ProblemSpec of a .inp file's lines; ``material(name)`` returns the
    volume material of a dispersive Volume_material_list entry, ``name``
    being the file name line as written (the reference opens name + '.vmat');
    ``open_file(name)`` returns the lines of an excitation function's data file;
    ``thin_layer(name, anisotropic)`` the thin layer of a dispersive surface
    material entry (the reference opens name + '.smat').

    ``mesh_file`` is the problem's NAME.mesh as the reference's mesher wrote
    it (``meshfile.read_mesh``).  With it the geometry is the mesher's, as
    the reference's solver takes it (MESH/read_mesh.F90): every volume is
    its cell list (any shape or rotation), the surface materials sit on
    their surfaces' face lists, the points on the mesh file's cells, and the
    PML volumes are checked against the PML packet.  Without it the reader
    voxelises the axis-aligned geometry itself."""
    packets = split_packets(lines)
    rec: Dict[str, Records] = {}
    for name, data in packets:
        if name in UNSUPPORTED:
            raise UnsupportedFeature(f"{name} packet: not supported by the GPU path")
        if name in NOT_READ:
            raise UnsupportedFeature(f"{name} packet: not read from .inp files; give the spec a ModeOutput")
        if name in rec:
            raise ValueError(f"{name} packet given twice")
        rec[name] = Records(name, data)
    skipped = [n for n, _ in packets if n in NEUTRAL]
    for need in ("mesh_outer_boundary_dimension", "simulation_time"):
        if need not in rec:
            raise ValueError(f"not a GGI_TLM problem file: no {need} packet")
    # the mesh, MESH/set_mesh_parameters.F90:40-100: a cell size wins over a cell count
    xmin, xmax, ymin, ymax, zmin, zmax = rec["mesh_outer_boundary_dimension"].values(6)
    ext = (xmax - xmin, ymax - ymin, zmax - zmin)
    if "mesh_cell_dimension" in rec:
        dl = rec["mesh_cell_dimension"].values(1)[0]
        n = tuple(max(1, nint(e / dl)) for e in ext)
    elif "mesh_dimensions_in_cells" in rec:
        nc = rec["mesh_dimensions_in_cells"].ints(3)
        # the division by 3 as a multiplication by 1/3, as the reference's build compiles it
        dl = (ext[0] / float(nc[0]) + ext[1] / float(nc[1]) + ext[2] / float(nc[2])) * (1.0 / 3.0)
        n = tuple(nint(e / dl) for e in ext)
    else:
        raise ValueError("neither Mesh_cell_dimension nor Mesh_dimensions_in_cells is given")
    if mesh_file is not None:  # the solver takes the mesh file's cell size and counts
        if tuple(mesh_file.n) != tuple(n) or abs(mesh_file.dl - dl) > 1e-9 * dl:
            raise ValueError(f"the mesh file's {mesh_file.n} cells of {mesh_file.dl} m do not match the problem "
                             f"file's {n} cells of {dl} m")
        dl = mesh_file.dl
    mesh = Mesh(xmin, ymin, zmin, dl, n)
    reduced_c = rec["reduced_c_factor"].values(1)[0] if "reduced_c_factor" in rec else 1.0
    if "bicubic_warp_flag" in rec and _logical(rec["bicubic_warp_flag"].line().split()[0]):
        raise UnsupportedFeature("bicubic frequency warping of the material filters")
    if "frequency_scale_flag" in rec:  # read_frequency_scale_flag.F90:53-54: a flag, then the scale
        r = rec["frequency_scale_flag"]
        r.line()
        if r.values(1)[0] != 1.0:  # s_to_z_warp (FILTER/filter_functions.F90:343-385) divides dt by it
            raise UnsupportedFeature("a frequency scale other than 1 for the material filters")
    dt = dl / (2.0 * C0 / reduced_c)  # TLM_SOLVER/set_TLM_solver_parameters.F90:93-95
    sim_time = rec["simulation_time"].values(1)[0]
    steps = nint(sim_time / dt)
    R = tuple(rec["outer_boundary_reflection_coefficient"].values(6)) \
        if "outer_boundary_reflection_coefficient" in rec else (0.0,) * 6
    spec = ProblemSpec(nx=n[0], ny=n[1], nz=n[2], dl=dl, n_timesteps=steps, R=R, origin=(xmin, ymin, zmin),
                       reduced_c=reduced_c, simulation_time=sim_time)
    if "wrapping_boundary_conditions" in rec:  # read_wrapping_boundary_conditions.F90:55-66
        w = rec["wrapping_boundary_conditions"].ints(3)
        if any(v not in (0, 1) for v in w):
            raise ValueError("wrapping_boundary_conditions packet: each flag is 1 or 0")
        spec.wrap = tuple(w)
    # PML, read_pml.F90:70-150: a line of six thicknesses (metres) or one for
    # all sides, the same for the reflection coefficients, then the order
    if "pml" in rec:
        r = rec["pml"]

        def six(line: str) -> List[float]:
            vals = []
            for tok in re.split(r"[\s,]+", line.strip()):
                try:
                    vals.append(fortran_real(tok))
                except ValueError:
                    break
            if not vals:
                raise ValueError(f"PML packet: no value on {line!r}")
            return vals[:6] if len(vals) >= 6 else vals[:1] * 6

        t, rr = six(r.line()), six(r.line())
        spec.pml_cells = tuple(nint(v / dl) for v in t)  # TLM_PML_volume_materials.F90:465
        spec.pml_r = tuple(rr)
        spec.pml_order = r.ints(1)[0]
    if mesh_file is not None and mesh_file.has_pml_section:
        if pml_cells_from_mesh(mesh_file) != tuple(spec.pml_cells):
            raise ValueError("the mesh file's PML volumes do not match the PML packet")
    # geometry, GEOMETRY/build_*.F90 with a translation only
    points: Dict[int, Tuple[float, float, float]] = {}
    if "point_list" in rec:
        r = rec["point_list"]
        for k in range(1, r.ints(1)[0] + 1):
            if r.ints(1)[0] != k:
                raise ValueError("Point_list packet: points must be numbered in order")
            p = r.values(3)
            tr = _transform(r, f"point {k}")
            points[k] = (p[0] + tr[0], p[1] + tr[1], p[2] + tr[2])
    def point_cell(pt: int) -> Tuple[int, int, int]:
        """The cell of a point: the mesh file's (problem_points(n)%cell), else get_cell_number."""
        if mesh_file is not None:
            if not 1 <= pt <= len(mesh_file.points):
                raise ValueError(f"point {pt} is not in the mesh file")
            return tuple(mesh_file.points[pt - 1].cell)
        return mesh.cell_of(points[pt])

    volumes = _geometry_list(rec["volume_list"], "volume", _VOLUME_PARAMS,
                             {"rectangular_block", "rectangular_block2"}) if "volume_list" in rec else {}
    surfaces = _geometry_list(rec["surface_list"], "surface", _SURFACE_PARAMS,
                              {"rectangular_block", "rectangular_block2", "rectangle", "xplane", "yplane",
                               "zplane"}) if "surface_list" in rec else {}

    def volume_block(v: int, what: str):
        if mesh_file is not None:  # the mesher's cells, whatever the volume's shape
            if not 1 <= v <= len(mesh_file.volumes):
                raise ValueError(f"{what}: volume {v} is not in the mesh file")
            cells = mesh_file.volumes[v - 1]
            check_cells(mesh_file, cells, f"volume {v}")
            return CellList(cells[:, :3])
        s = volumes[v]
        if s.rotated:
            raise UnsupportedFeature(f"{what} on a rotated {s.kind}: only zero Euler angles are supported")
        if s.par is None:
            raise UnsupportedFeature(f"{what} on a volume of type {s.kind!r}")
        return _block_cells(mesh, s.par, s.tr, s.kind)

    def mode_faces(surf: int, side: int, name: str, cols: Sequence[int], what: str):
        """The faces of a mode excitation or output and their mode field
        (set_mode_excitations_in_mesh, mode_excitation.F90:35-250, and
        set_mode_outputs_in_mesh, output_modes.F90:35-250): the mode file's
        samples in file order, moved by the offset between the bounding
        cells of the samples and of the surface's faces, each on the
        surface's (single) face code, taken from the other side of the face
        unless ``side`` is 1."""
        if open_file is None:
            raise UnsupportedFeature(f"{what} from the mode file {name!r}: no file opener")
        xcol, ycol, zcol, mcol = cols
        if sorted((xcol, ycol, zcol)) != [1, 2, 3] or mcol < 4:
            raise ValueError(f"{what}: mode file columns {cols} (x, y, z among 1..3, the data column above 3)")
        samples = []
        for ln in open_file(name):
            f = ln.replace(",", " ").split()
            if not f:
                continue
            if len(f) < mcol:
                raise ValueError(f"{what}: mode file {name!r}: a line with fewer than {mcol} values")
            c = (int(f[0]), int(f[1]), int(f[2]))
            samples.append(((c[xcol - 1], c[ycol - 1], c[zcol - 1]), fortran_real(f[mcol - 1])))
        geo, orient = surface_geo(surf, what, 1)
        faces = FarFieldSurface([], side=orient, **geo).faces()  # the surface's own face list
        if not faces or not samples:
            return []
        codes = {code for _, code in faces}
        if len(codes) != 1:
            raise ValueError(f"{what}: surface {surf} has faces of more than one orientation")
        code = codes.pop()
        lo_s = [min(c[a] for c, _ in faces) for a in range(3)]
        hi_s = [max(c[a] for c, _ in faces) for a in range(3)]
        lo_m = [min(c[a] for c, _ in samples) for a in range(3)]
        hi_m = [max(c[a] for c, _ in samples) for a in range(3)]
        n_s = [h - l + 1 for l, h in zip(lo_s, hi_s)]
        n_m = [h - l + 1 for l, h in zip(lo_m, hi_m)]
        if n_s != n_m:
            raise ValueError(f"{what}: the mode's extent {n_m} differs from surface {surf}'s {n_s}")
        if n_m[(code - 1) % 3] != 1:
            raise ValueError(f"{what}: the mode is not planar along its surface's normal")
        off = [a - b for a, b in zip(lo_s, lo_m)]
        flip = {1: (0, -1, 4), 2: (1, -1, 5), 3: (2, -1, 6), 4: (0, 1, 1), 5: (1, 1, 2), 6: (2, 1, 3)}
        out = []
        for c, field in samples:
            cell, fc = [c[a] + off[a] for a in range(3)], code
            if side != 1:  # the face seen from the neighbouring cell
                ax, d, fc = flip[code]
                cell[ax] += d
            out.append((tuple(cell), fc, field))
        return out

    def surface_geo(surf: int, what: str, side: int) -> Tuple[dict, int]:
        """box=, plane= or (with a mesh file) records= of a surface, and the
        side in the spec's convention: the packet's side times the plane's
        orientation, or the packet's side for the mesh file's own faces."""
        if mesh_file is not None:
            if not 1 <= surf <= len(mesh_file.surfaces):
                raise ValueError(f"{what}: surface {surf} is not in the mesh file")
            f = mesh_file.surfaces[surf - 1].faces
            if f.size and (f[:, 3].min() < 1 or f[:, 3].max() > 6):
                raise ValueError(f"{what}: surface {surf} lists a face code outside 1..6")
            return dict(records=[((int(i), int(j), int(k)), int(c)) for i, j, k, c in f.tolist()]), side
        return _surface_geo(mesh, surfaces[surf], what, side)

    # volume materials, read_volume_material_list.F90:90-180
    if "volume_material_list" in rec:
        r = rec["volume_material_list"]
        for k in range(1, r.ints(1)[0] + 1):
            if r.ints(1)[0] != k:
                raise ValueError("Volume_material_list packet: materials must be numbered in order")
            kind = r.text()
            if kind == "dispersive":
                mat = material(r.line().strip())
            elif kind in ("pec", "pmc"):
                mat = VolumeMaterial(type=MAT_PEC if kind == "pec" else MAT_PMC)
            else:
                raise ValueError(f"Volume_material_list packet: unknown material type {kind!r}")
            spec.materials.append(mat)
            nv = r.ints(1)[0]
            for v in r.ints(nv):
                spec.material_regions.append((k, volume_block(v, "a volume material")))
    # excitation functions, read_excitation_function_list.F90:92-250; a
    # name that is no function type is a data file of samples
    if "excitation_function_list" in rec:
        r = rec["excitation_function_list"]
        for k in range(1, r.ints(1)[0] + 1):
            if r.ints(1)[0] != k:
                raise ValueError("Excitation_function_list packet: functions must be numbered in order")
            raw = r.line()
            kind = raw.rstrip().lower()
            if kind in _N_PARAMS:
                spec.functions.append(ExcitationFunction(kind, tuple(r.values(_N_PARAMS[kind]))))
            elif kind in _OTHER_FUNCTIONS:
                raise UnsupportedFeature(f"excitation function {kind!r}")
            else:
                if open_file is None:
                    raise UnsupportedFeature(f"excitation function from the file {raw.strip()!r}: no file opener")
                n_ignore, n_time, n_value = r.ints(1)[0], r.ints(1)[0], r.ints(1)[0]
                samples = _samples(open_file(raw.strip()), n_ignore, n_time, n_value)
                spec.functions.append(ExcitationFunction("file", tuple(r.values(2)), samples))
    # point excitations, read_excitation_point_list.F90:75-110
    if "excitation_point_list" in rec:
        r = rec["excitation_point_list"]
        for k in range(1, r.ints(1)[0] + 1):
            if r.ints(1)[0] != k:
                raise ValueError("Excitation_point_list packet: points must be numbered in order")
            fn, pt = r.ints(1)[0], r.ints(1)[0]
            comp = _component(r, _FIELD_OR_CURRENT)
            face = _face(r)
            kind = r.text()
            if kind not in ("soft", "hard"):
                raise ValueError(f"Excitation_point_list packet: source type {kind!r}")
            spec.point_excitations.append(PointExcitation(point_cell(pt), comp, fn,
                                                          SOURCE_SOFT if kind == "soft" else SOURCE_HARD, face=face))
    # excitation surfaces and volumes (read_excitation_surface_list.F90:66-120,
    # read_excitation_volume_list.F90): Surface_excitation and Volume_excitation
    # (excitation_surfaces.F90, excitation_volumes.F90) add the function's value
    # on every face side / cell of the geometry to the same field tables as the
    # excitation points, after them, so each face side or cell becomes a face
    # or centre point excitation appended after the packet's points
    if "excitation_surface_list" in rec:
        r = rec["excitation_surface_list"]
        for k in range(1, r.ints(1)[0] + 1):
            if r.ints(1)[0] != k:
                raise ValueError("Excitation_surface_list packet: surfaces must be numbered in order")
            fn, surf, side = r.ints(1)[0], r.ints(1)[0], r.ints(1)[0]
            if side not in (1, -1, 0):
                raise ValueError("Excitation_surface_list packet: the side must be 1, -1 or 0")
            comp = _component(r, _FIELD)
            kind = r.text()
            if kind not in ("soft", "hard"):
                raise ValueError(f"Excitation_surface_list packet: source type {kind!r}")
            # side 0 takes each face from the other side (as -1) and excites both of its sides;
            # otherwise the side of the face the (possibly flipped) face code names
            geo, eff = surface_geo(surf, "an excitation surface", -1 if side == 0 else side)
            for cell, code in FarFieldSurface([], side=eff, **geo).faces():
                spec.point_excitations.append(PointExcitation(
                    tuple(cell), comp, fn, SOURCE_SOFT if kind == "soft" else SOURCE_HARD,
                    face=_FACE_OF_CODE[code], one_side=side != 0))
    if "excitation_volume_list" in rec:
        r = rec["excitation_volume_list"]
        for k in range(1, r.ints(1)[0] + 1):
            if r.ints(1)[0] != k:
                raise ValueError("Excitation_volume_list packet: volumes must be numbered in order")
            fn, v = r.ints(1)[0], r.ints(1)[0]
            comp = _component(r, _FIELD)
            kind = r.text()
            if kind not in ("soft", "hard"):
                raise ValueError(f"Excitation_volume_list packet: source type {kind!r}")
            region = volume_block(v, "an excitation volume")
            zz, yy, xx = np.nonzero(FrequencyOutputVolume(region, [], comp).mask(spec))
            for x, y, z in zip(xx, yy, zz):  # the volume's cells in traversal order
                spec.point_excitations.append(PointExcitation(
                    (int(x) + 1, int(y) + 1, int(z) + 1), comp, fn, SOURCE_SOFT if kind == "soft" else SOURCE_HARD))
    # mode excitations (read_excitation_mode_list.F90:52-110, Mode_excitation,
    # mode_excitation.F90:330-420): the function's value times each face's
    # mode field on one side of the face, or half of it on both sides for
    # side 0 (E and H only: the Huygens surface's J, M, added before them in
    # the step, touch other components)
    if "excitation_mode_list" in rec:
        r = rec["excitation_mode_list"]
        for k in range(1, r.ints(1)[0] + 1):
            if r.ints(1)[0] != k:
                raise ValueError("Excitation_mode_list packet: modes must be numbered in order")
            fn, surf, side = r.ints(1)[0], r.ints(1)[0], r.ints(1)[0]
            if side not in (1, -1, 0):
                raise ValueError("Excitation_mode_list packet: the side must be 1, -1 or 0")
            comp = _component(r, _FIELD)
            kind = r.text()
            if kind not in ("soft", "hard"):
                raise ValueError(f"Excitation_mode_list packet: source type {kind!r}")
            name = r.line().strip()
            cols = [r.ints(1)[0] for _ in range(4)]
            for cell, code, field in mode_faces(surf, side, name, cols, "an excitation mode"):
                spec.point_excitations.append(PointExcitation(
                    cell, comp, fn, SOURCE_SOFT if kind == "soft" else SOURCE_HARD, face=_FACE_OF_CODE[code],
                    one_side=side != 0, scale=field if side != 0 else field / 2.0))
    # mode outputs (read_output_mode_list.F90:50-90, Mode_output,
    # output_modes.F90:546-620)
    if "output_mode_list" in rec:
        r = rec["output_mode_list"]
        for k in range(1, r.ints(1)[0] + 1):
            if r.ints(1)[0] != k:
                raise ValueError("Output_mode_list packet: modes must be numbered in order")
            surf, side = r.ints(1)[0], r.ints(1)[0]
            if side not in (1, -1):
                raise ValueError("Output_mode_list packet: the side must be 1 or -1")
            comp = _component(r, _FIELD)
            name = r.line().strip()
            cols = [r.ints(1)[0] for _ in range(4)]
            spec.mode_outputs.append(ModeOutput(comp, None, None, samples=mode_faces(surf, side, name, cols,
                                                                                      "an output mode")))
    # the Huygens surface, read_huygens_surface.F90:89-200
    if "huygens_surface" in rec:
        r = rec["huygens_surface"]
        surf, side = r.ints(1)[0], r.ints(1)[0]
        if side not in (1, -1):
            raise ValueError("Huygens_surface packet: the side must be 1 or -1")
        z0 = Z0
        if r.peek_text() == "wave_impedance":
            r.line()
            z0 = r.values(1)[0]
        fn = r.ints(1)[0]
        angles = []
        for _ in range(2):  # '(A1)': a line starting with r or R asks for a random choice
            if r.pos < len(r.lines) and r.lines[r.pos][:1] in ("r", "R"):
                raise UnsupportedFeature("random Huygens wave direction or polarisation")
            angles += r.values(2)
        kt, kp, et, ep = angles
        if surf == 0:
            spec.huygens = HuygensOuter(fn, kt, kp, et, ep, wave_impedance=z0)
        else:
            kind, g, orient = _surface_cells(mesh, surfaces[surf], "a Huygens surface")
            if kind == "box":
                spec.huygens = HuygensBox(g[0], g[1], g[2], fn, kt, kp, et, ep, side=side, wave_impedance=z0)
            else:
                spec.huygens = HuygensPlane(g[0], g[1], g[2], g[3], fn, kt, kp, et, ep, side=side * orient,
                                            wave_impedance=z0)
    # output points, read_output_point_list.F90:85-125
    timing: List[Optional[Tuple[int, int, int]]] = []
    if "output_point_list" in rec:
        r = rec["output_point_list"]
        for k in range(1, r.ints(1)[0] + 1):
            if r.ints(1)[0] != k:
                raise ValueError("Output_point_list packet: points must be numbered in order")
            pt = r.ints(1)[0]
            comp = _component(r, _FIELD)
            spec.outputs.append(OutputPoint(point_cell(pt), comp, _face(r)))
            timing.append(_timing(r, dt))
    # output surfaces, read_output_surface_list.F90:88-135: side 1, -1, or 0
    # (J from both sides, on the faces of side -1)
    if "output_surface_list" in rec:
        r = rec["output_surface_list"]
        for k in range(1, r.ints(1)[0] + 1):
            if r.ints(1)[0] != k:
                raise ValueError("Output_surface_list packet: surfaces must be numbered in order")
            surf, side = r.ints(1)[0], r.ints(1)[0]
            if side not in (1, -1, 0):
                raise ValueError("Output_surface_list packet: the side must be 1, -1 or 0")
            comp = _component(r, _SURFACE_FIELD, width=2)
            if side == 0 and comp not in ("Jx", "Jy", "Jz", "Jm"):
                raise ValueError("Output_surface_list packet: output on both sides is for Jx, Jy, Jz, Jmagnitude")
            geo, eff = surface_geo(surf, "an output surface", -1 if side == 0 else side)
            spec.output_surfaces.append(OutputSurface(comp, side=eff, both_sides=side == 0,
                                                      **geo, **_steps(_timing(r, dt))))
    # output volumes, read_output_volume_list.F90:85-105
    if "output_volume_list" in rec:
        r = rec["output_volume_list"]
        for k in range(1, r.ints(1)[0] + 1):
            if r.ints(1)[0] != k:
                raise ValueError("Output_volume_list packet: volumes must be numbered in order")
            v = r.ints(1)[0]
            comp = _component(r, _FIELD)
            spec.output_volumes.append(OutputVolume(volume_block(v, "an output volume"), comp, "field",
                                                    **_steps(_timing(r, dt))))
    _read_outputs(rec, mesh, dt, spec, surface_geo, volume_block, post := {})
    if "surface_material_list" in rec:
        _read_surface_materials(rec["surface_material_list"], mesh, spec, surfaces, mesh_file, thin_layer)
    if "set_small_to_zero" in rec:  # read_small_to_zero.F90:55-59
        r = rec["set_small_to_zero"]
        spec.small_to_zero = (r.ints(1)[0], r.values(1)[0])
    return InpProblem(spec, skipped, timing, post)


def _side(r: Records, allowed=(1, -1)) -> int:
    side = r.ints(1)[0]
    if side not in allowed:
        raise ValueError(f"{r.name} packet: the side must be one of {allowed}")
    return side


def _surface_geo(mesh: Mesh, s: Shape, what: str, side: int) -> Tuple[dict, int]:
    """The box= or plane= argument of a spec surface and the side in the
    spec's convention (the packet's side times the plane's orientation)."""
    kind, g, orient = _surface_cells(mesh, s, what)
    return (dict(box=g) if kind == "box" else dict(plane=g)), side * orient


def _numbered(r: Records, what: str):
    n = r.ints(1)[0]
    for k in range(1, n + 1):
        if r.ints(1)[0] != k:
            raise ValueError(f"{r.name} packet: {what} must be numbered in order")
        yield k


def _read_outputs(rec: Dict[str, Records], mesh: Mesh, dt: float, spec: ProblemSpec,
                  surface_geo: Callable[[int, str, int], Tuple[dict, int]], volume_block: Callable[[int, str], object],
                  post: dict) -> None:
    """The volume and surface output packets other than Output_volume_list
    and Output_surface_list, each entry becoming one spec entry (one
    frequency per entry, as the reference stores them)."""
    for name, kind in (("output_volume_average_list", "average"), ("output_volume_peak_list", "peak")):
        if name in rec:  # read_output_volume_average_list.F90:78-100 / read_output_volume_peak_list.F90:78-100
            r = rec[name]
            for _ in _numbered(r, "volumes"):
                v = r.ints(1)[0]
                comp = _component(r, _FIELD)
                spec.output_volumes.append(OutputVolume(volume_block(v, f"an output volume {kind}"), comp, kind,
                                                        **_steps(_timing(r, dt))))
    if "frequency_output_volume_list" in rec and "frequency_output_volume_list_xyz" in rec:
        raise ValueError("frequency_output_volume_list and frequency_output_volume_list_xyz both given")
    for name in ("frequency_output_volume_list", "frequency_output_volume_list_xyz"):
        if name in rec:  # read_frequency_output_volume.F90:77-160
            r = rec[name]
            n = r.ints(1)[0]
            every = 1
            if name.endswith("_xyz") and r.peek_text(80)[:12] == "output_every":
                every = int(fortran_real(r.line()[12:].split()[0]))
            for k in range(1, n + 1):
                if r.ints(1)[0] != k:
                    raise ValueError(f"{name} packet: volumes must be numbered in order")
                v = r.ints(1)[0]
                freq = r.values(1)[0]
                comp = _component(r, _FIELD)
                spec.frequency_output_volumes.append(FrequencyOutputVolume(
                    volume_block(v, "a frequency output volume"), [freq], comp, every=every,
                    **_steps(_timing(r, dt))))
    if "frequency_output_surface_list" in rec:  # read_frequency_output_surface.F90:63-125
        r = rec["frequency_output_surface_list"]
        for _ in _numbered(r, "surfaces"):
            surf, side = r.ints(1)[0], _side(r)
            freq = r.values(1)[0]
            comp = _component(r, _FIELD_OR_CURRENT, width=2)
            geo, eff = surface_geo(surf, "a frequency output surface", side)
            t = _timing(r, dt)
            if "box" in geo:
                raise UnsupportedFeature("frequency output surface on a closed box: planar patches or a mesh "
                                         "file's faces only")
            gate = _steps(t)  # the surface's output steps (get_output_flag)
            if "plane" in geo:
                ax, ix, r0, r1 = geo["plane"]
                spec.dft_surfaces.append(DFTSurface(ax, ix, r0, r1, [freq], comp, side=eff, **gate))
            else:
                spec.dft_surfaces.append(DFTSurface(0, 0, (0, 0), (0, 0), [freq], comp, side=eff,
                                                    records=geo["records"], **gate))
    if "far_field_surface_list" in rec:  # read_far_field_surface.F90:79-165
        r = rec["far_field_surface_list"]
        post["far_field"] = []
        for _ in _numbered(r, "surfaces"):
            surf, side = r.ints(1)[0], _side(r)
            freq = r.values(1)[0]
            theta, phi = tuple(r.values(3)), tuple(r.values(3))
            dim = 3
            if r.peek_text(2) == "2d":  # the optional 2D transform, about z only
                r.line()
                if r.text() != "z":
                    raise ValueError("far_field_surface_list packet: a 2D transform about z only")
                dim, theta = 2, (90.0, 90.0, 180.0 / 3.141592653589793)  # theta pi/2 with a 1 rad step
            geo, eff = surface_geo(surf, "a far-field surface", side)
            spec.far_field_surfaces.append(FarFieldSurface([freq], side=eff, **geo))
            post["far_field"].append(dict(frequency=freq, theta=theta, phi=phi, dim=dim))
    if "rcs_surface" in rec:  # read_rcs_surface.F90:63-85
        r = rec["rcs_surface"]
        surf, side = r.ints(1)[0], _side(r)
        post["rcs"] = tuple(r.values(3))  # fmin, fmax, fstep
        theta, phi = r.values(1)[0], r.values(1)[0]
        geo, eff = surface_geo(surf, "an RCS surface", side)
        spec.rcs_surface = RCSSurface(theta, phi, side=eff, **geo)
    if "frequency_domain_power_surface_list" in rec:  # read_frequency_domain_power_surface.F90:63-105
        r = rec["frequency_domain_power_surface_list"]
        n_first = None
        for _ in _numbered(r, "surfaces"):
            surf, side = r.ints(1)[0], _side(r)
            fmin, fmax, nf = r.values(3)
            nf = int(nf)
            if n_first is not None and nf != n_first:
                raise ValueError("frequency_domain_power_surface_list packet: the surfaces must have the same "
                                 "number of frequencies")
            n_first = nf
            fstep = (fmax - fmin) / float(nf - 1) if nf != 1 else 0.0
            freqs = [fmin + (k - 1) * fstep for k in range(1, nf + 1)]  # frequency_domain_power_surfaces.F90:328
            geo, eff = surface_geo(surf, "a power surface", side)
            spec.power_surfaces.append(PowerSurface(freqs, side=eff, **geo))
    if "sar_volume_list" in rec:  # read_SAR_volume_list.F90:69-90: material number, frequency, density
        r = rec["sar_volume_list"]
        post["sar_density"] = []
        for _ in _numbered(r, "volumes"):
            m = r.ints(1)[0]
            freq, rho = r.values(1)[0], r.values(1)[0]
            spec.sar_volumes.append(SARVolume(_material_block(spec, m), [freq]))
            post["sar_density"].append(rho)


def _material_block(spec: ProblemSpec, m: int):
    """The cells of volume material ``m`` (SAR_volumes.F90:62-95 takes every
    cell whose material is m) when they form one region (a block, or a mesh
    file's cell list) that no other material overlaps."""
    own = [b for k, b in spec.material_regions if k == m]
    if len(own) != 1:
        raise UnsupportedFeature("a SAR volume on a material of several volumes")
    b = own[0]
    mine = _region_mask(spec, b)
    for k, o in spec.material_regions:
        if k != m and np.any(mine & _region_mask(spec, o)):
            raise UnsupportedFeature("a SAR volume on a material that another material overlaps")
    return b


def _read_surface_materials(r: Records, mesh: Mesh, spec: ProblemSpec, surfaces: Dict[int, Shape],
                            mesh_file: Optional[MeshFile] = None,
                            thin_layer: Optional[Callable[[str, bool], SurfaceMaterial]] = None) -> None:
    """read_surface_material_list.F90:111-470 for PEC, PMC, free-space and
    dispersive (isotropic or anisotropic thin-layer) surfaces: number, type,
    for a thin layer the name of its .smat file, the number of surfaces,
    their numbers and their orientations (+1 or -1).  A box surface becomes
    its six boundary planes; with a mesh file every surface is its face
    list, whatever its shape.  ``thin_layer(name, anisotropic)`` returns the
    layer a .smat file describes.

    A thin layer's orientation matters: set_surface_material_mesh
    (TLM_surface_materials.F90:150-175) gives each face the orientation's
    sign when the surface records the face as the min face of a cell and the
    opposite sign when it records it as the max face of the cell below."""
    names = {"pec": "PEC", "pmc": "PMC", "free_space": "free", "dispersive": "dispersive",
             "anisotropic_dispersive": "dispersive"}
    for _ in _numbered(r, "surface materials"):
        kind = r.text()
        if kind not in names:
            raise UnsupportedFeature(f"surface material {kind!r}: only PEC, PMC, free-space and dispersive "
                                     "surfaces")
        material = 0
        if names[kind] == "dispersive":
            name = r.line().strip()
            if thin_layer is None:
                raise UnsupportedFeature(f"thin-layer material {name!r}: no surface material file resolver")
            spec.thin_layers.append(thin_layer(name, kind == "anisotropic_dispersive"))
            material = len(spec.thin_layers)
        n = r.ints(1)[0]
        nums = r.ints(n)
        signs = r.ints(n)
        if any(v not in (1, -1) for v in signs):
            raise ValueError("surface_material_list packet: orientations must be +1 or -1")
        for num, sg in zip(nums, signs):
            if mesh_file is not None:
                if not 1 <= num <= len(mesh_file.surfaces):
                    raise ValueError(f"surface {num} is not in the mesh file")
                rec = mesh_file.surfaces[num - 1].faces
                faces = connect_faces(mesh_file, rec, f"surface {num}")
                fs = [sg if code <= 3 else -sg for code in rec[:, 3].tolist()]
                spec.surface_sheets.append(SurfaceSheet(names[kind], 0, 0, (0, 0), (0, 0), faces=faces,
                                                        material=material, sign=fs))
                continue
            geo, orient = _surface_geo(mesh, surfaces[num], "a surface material", 1)
            if "plane" in geo:
                ax, ix, r0, r1 = geo["plane"]
                spec.surface_sheets.append(SurfaceSheet(names[kind], ax, ix, r0, r1, material=material,
                                                        sign=sg * orient))
            else:
                (i0, i1), (j0, j1), (k0, k1) = geo["box"]
                # the block's faces sit on the outside cells: max faces of the cells before its min
                # planes, min faces of the cells past its max planes
                for ax, ix, r0, r1, rs in ((1, i0 - 1, (j0, j1), (k0, k1), -1), (1, i1, (j0, j1), (k0, k1), 1),
                                           (2, j0 - 1, (i0, i1), (k0, k1), -1), (2, j1, (i0, i1), (k0, k1), 1),
                                           (3, k0 - 1, (i0, i1), (j0, j1), -1), (3, k1, (i0, i1), (j0, j1), 1)):
                    spec.surface_sheets.append(SurfaceSheet(names[kind], ax, ix, r0, r1, material=material,
                                                            sign=sg * rs))


# the packets that only ask for results; read_inp_lenient may leave them out
OUTPUT_PACKETS = {"output_point_list", "output_surface_list", "output_volume_list", "output_volume_average_list",
                  "output_volume_peak_list", "frequency_output_volume_list", "frequency_output_volume_list_xyz",
                  "frequency_output_surface_list", "far_field_surface_list", "rcs_surface",
                  "frequency_domain_power_surface_list", "sar_volume_list", "output_mode_list"}


def read_inp_lenient(lines: Sequence[str], material: Callable[[str], VolumeMaterial],
                     open_file: Optional[Callable[[str], Sequence[str]]] = None,
                     mesh_file: Optional[MeshFile] = None,
                     thin_layer: Optional[Callable[[str, bool], SurfaceMaterial]] = None) -> InpProblem:
    """read_inp, leaving out each output packet that read_inp refuses (a
    result the GPU path cannot produce exactly, such as an output surface on
    rotated geometry) and listing it in ``skipped`` as "<packet>: <reason>".
    Everything else is read as strictly as read_inp reads it."""
    packets = split_packets(lines)

    def text(keep):
        out = []
        for name, data in packets:
            if name in keep:
                out.append(name)
                out.extend(data)
        return out

    core = {n for n, _ in packets if n not in OUTPUT_PACKETS}
    dropped = []
    for name in [n for n, _ in packets if n in OUTPUT_PACKETS]:
        try:
            read_inp(text(core | {name}), material, open_file, mesh_file, thin_layer)
        except UnsupportedFeature as e:
            dropped.append(f"{name}: {e}")
    keep = core | {n for n, _ in packets if n in OUTPUT_PACKETS and not any(d.startswith(n + ":") for d in dropped)}
    p = read_inp(text(keep), material, open_file, mesh_file, thin_layer)
    p.skipped.extend(dropped)
    return p


def vmat_in(directory: str) -> Callable[[str], VolumeMaterial]:
    """A material resolver reading ``<directory>/<name>.vmat``."""
    from .vmat import read_vmat

    return lambda name: read_vmat(os.path.join(directory, name + ".vmat"))


def smat_in(directory: str) -> Callable[[str, bool], SurfaceMaterial]:
    """A thin-layer resolver reading ``<directory>/<name>.smat``."""
    from .smat import read_smat

    return lambda name, anisotropic: read_smat(os.path.join(directory, name + ".smat"), anisotropic)


def read_inp_file(path: str, material: Optional[Callable[[str], VolumeMaterial]] = None,
                  lenient: bool = False, mesh: Optional[bool] = None) -> InpProblem:
    """read_inp (read_inp_lenient with ``lenient``) of a file; material and
    data file names resolve against the file's directory unless ``material``
    is given.  The text is read as Latin-1: the reference's inputs hold stray
    non-ASCII bytes in remarks.  The mesh file NAME.mesh beside NAME.inp,
    when there is one (or when ``mesh`` is True), gives the geometry, as it
    does to the reference's solver; ``mesh=False`` voxelises the .inp
    geometry instead."""
    directory = os.path.dirname(os.path.abspath(path))
    with open(path, encoding="latin-1") as f:
        lines = f.read().splitlines()
    mesh_path = os.path.splitext(path)[0] + ".mesh"
    mesh_file = None
    if mesh or (mesh is None and os.path.exists(mesh_path)):
        with open(mesh_path, encoding="latin-1") as f:
            mesh_file = read_mesh(f.read().splitlines())

    def open_file(name: str) -> List[str]:
        with open(os.path.join(directory, name), encoding="latin-1") as g:
            return g.read().splitlines()

    return (read_inp_lenient if lenient else read_inp)(lines, material or vmat_in(directory), open_file, mesh_file,
                                                      smat_in(directory))
