"""Host-side problem setup: builds the tables GGI_TLM's setup stage leaves in
its modules before ``run_TLM`` is called (SRC/GGI_TLM.F90:100-154).

This is the part of the reference that stays on the host (layer L3): mesh
parameters, cell update codes, volume-material Z-filter coefficients, the PML
parameter table, excitation-function tables, Huygens-surface data, output
points and frequency-domain output surfaces.  The same tables feed both the
GPU path (through the C-ABI in ``include/tlm_gpu.h``) and the CPU oracle.

Geometry is restricted to what the hot path needs and what can be voxelised
exactly without the reference's triangle/tet mesher: axis-aligned blocks and
spheres (cell-centre-inside test), planar Huygens patches and planar output
patches on cell faces, point sources and point probes at cell centres.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

# SRC/CONSTANTS/constants.F90:27-39
PI = 3.141592653589793
Z0 = 376.73031346177
Y0 = 1.0 / Z0
EPS0 = 8.8541878176e-12
MU0 = 3.141592653589793 * 4e-7
C0 = 2.99792458e8

MAX_ORDER = 8  # max Z-filter order carried in the coefficient tables

# field components, SRC/TLM_MODULES/TLM_Modules.F90:164-176
COMPONENTS = {"Ex": 1, "Ey": 2, "Ez": 3, "Hx": 4, "Hy": 5, "Hz": 6, "Jx": 7, "Jy": 8, "Jz": 9,
              "Mx": 10, "My": 11, "Mz": 12}
# a point on a cell face -> (offset of the cell whose min face it is, axis, side 1/2),
# get_min_face (MESH/general_mesh_subroutines.F90) and the side rule of
# excitation_points.F90:295-307 / output_points.F90:386-399
FACE_POINT = {"xmin": ((0, 0, 0), 1, 1), "xmax": ((1, 0, 0), 1, 2), "ymin": ((0, 0, 0), 2, 1),
              "ymax": ((0, 1, 0), 2, 2), "zmin": ((0, 0, 0), 3, 1), "zmax": ((0, 0, 1), 3, 2)}
# faces, SRC/TLM_MODULES/Mesh_Modules.F90:40-46
FACE_XMIN, FACE_YMIN, FACE_ZMIN, FACE_XMAX, FACE_YMAX, FACE_ZMAX, CENTRE = 1, 2, 3, 4, 5, 6, 7
# volume material types, SRC/TLM_MODULES/TLM_material_modules.F90:72-78
MAT_PEC, MAT_PMC, MAT_DISPERSIVE = 1, 2, 3
SOURCE_HARD, SOURCE_SOFT = 0, 1  # TLM_excitation_modules.F90:162-163


class UnsupportedFeature(ValueError):
    """A feature outside the GPU path (cables, Ngspice, thin layers, ...)."""


def nint(x: float) -> int:
    """Fortran NINT: round half away from zero."""
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


# ---------------------------------------------------------------------------
# Filters (SRC/FILTER)
# ---------------------------------------------------------------------------
@dataclass
class Sfilter:
    """Laplace-domain rational filter a(s/wnorm)/b(s/wnorm), FILTER/filter_types.F90:37-43."""

    wnorm: float
    a: List[float]
    b: List[float]


def _poly_mul(p: Sequence[float], q: Sequence[float]) -> List[float]:
    out = [0.0] * (len(p) + len(q) - 1)
    for i, pi in enumerate(p):
        for j, qj in enumerate(q):
            out[i + j] = out[i + j] + pi * qj
    return out


def _findroots(coeff: Sequence[float]) -> List[complex]:
    """Roots of a polynomial via the eigenvalues of its companion (upper
    Hessenberg) matrix, POLYNOMIAL/root_finding.F90:40-100.  The reference
    calls EISPACK hqr; numpy's LAPACK eigensolver returns the same roots to
    rounding (~1e-16 relative)."""
    n = len(coeff) - 1
    if n <= 0:
        return []
    h = np.zeros((n, n))
    for i in range(n):
        h[0, i] = -coeff[n - 1 - i] / coeff[n]
        if i != n - 1:
            h[i + 1, i] = 1.0
    w = np.linalg.eigvals(h)
    roots = []
    for r in w:
        wr, wi = float(r.real), float(r.imag)
        if abs(wi) <= abs(1e-10 * wr):
            wi = 0.0
        roots.append(complex(wr, wi))
    return roots


def _rootsort(roots: List[complex]) -> Tuple[List[complex], List[complex]]:
    """Split roots into real roots and conjugate-paired complex roots,
    POLYNOMIAL/root_finding.F90:135-230."""
    rroots, croots = [], []
    for r in roots:
        if abs(r) == 0.0 or abs((r * complex(0, -1)).real) / abs(r) <= 1e-8:
            rroots.append(r)
        else:
            croots.append(r)
    ncomplex = len(croots) // 2
    for i in range(ncomplex):
        fpair = 2 * i
        c0 = croots[fpair]
        tangle = abs((complex(0, -1) * c0 / c0.real).real) if c0.real != 0.0 else 1e10
        for k in range(fpair + 1, 2 * ncomplex):
            ssum = croots[fpair] + croots[k]
            tanglesum = abs((complex(0, -1) * ssum / abs(ssum)).real) if abs(ssum) != 0.0 else 0.0
            if tanglesum / tangle < 1e-5:
                croots[fpair + 1], croots[k] = croots[k], croots[fpair + 1]
    return rroots, croots[: 2 * ncomplex]


def _trim(coeff: Sequence[float]) -> List[float]:
    """Order reduction used at the start of bilinear_s_to_z
    (filter_subroutines.F90:640-660): the order stays the declared one if any
    coefficient is non-zero, else it drops to 0."""
    if any(c != 0.0 for c in coeff):
        return list(coeff)
    return [coeff[0]]


def bilinear_s_to_z(fs: Sfilter, dt: float) -> Tuple[List[float], List[float]]:
    """Bilinear s->z transform, FILTER/filter_subroutines.F90:601-886.
    Returns (a, b) coefficients of the z^-1 polynomials with b[0]=1."""
    a_s = _trim(fs.a)
    b_s = _trim(fs.b)
    aorder, border = len(a_s) - 1, len(b_s) - 1
    max_order = max(aorder, border)
    dt2 = 2.0 / (dt * fs.wnorm)
    roots = _findroots(a_s)
    poles = _findroots(b_s)
    if b_s[border] == 0.0:
        raise ValueError("bilinear_s_to_z: zero leading denominator coefficient")
    gain = a_s[aorder] / b_s[border]
    zpolys = []
    for loop, rts in ((1, roots), (2, poles)):
        rr, cr = _rootsort(rts)
        a = [1.0]
        for i in range(len(cr) // 2):
            modc = (cr[2 * i] * cr[2 * i + 1]).real
            rec2 = (cr[2 * i] + cr[2 * i + 1]).real
            b2 = [dt2 * dt2 - rec2 * dt2 + modc, -2.0 * dt2 * dt2 + 2.0 * modc, dt2 * dt2 + rec2 * dt2 + modc]
            a = _poly_mul(a, b2)
        for r in rr:
            b1 = [dt2 - r.real, -dt2 - r.real]
            a = _poly_mul(a, b1)
        zpolys.append(a)
    znum = [c * gain for c in zpolys[0]]
    zden = list(zpolys[1])
    ztemp = [1.0, 1.0]
    if aorder > border:
        for _ in range(aorder - border):
            zden = _poly_mul(zden, ztemp)
    elif border > aorder:
        for _ in range(border - aorder):
            znum = _poly_mul(znum, ztemp)
    b0 = zden[0]
    if b0 != 0.0:
        znum = [c / b0 for c in znum[: max_order + 1]]
        zden = [c / b0 for c in zden[: max_order + 1]]
    return znum, zden


def z_fast_slow_decomposition(a: List[float], b: List[float]) -> Tuple[float, List[float], List[float]]:
    """FILTER/filter_subroutines.F90:1145-1213."""
    if len(a) != len(b):
        raise ValueError("Z_fast_slow_decomposition: aorder != border")
    f_fast = a[0] / b[0]
    out = list(a)
    out[0] = 0.0
    for i in range(1, len(b)):
        out[i] = out[i] - b[i] * f_fast
    return f_fast, out, list(b)


def electric_susceptibility_impedance(eps: Sfilter, K: float) -> Sfilter:
    """Z(s)=1/(s*K*(eps_r(s)-1)), FILTER/filter_subroutines.F90:1379-1431."""
    border = len(eps.a) - 1 + 1
    bc = [0.0] * (border + 1)
    for i, c in enumerate(eps.a):
        bc[i + 1] = K * eps.wnorm * c
    for i, c in enumerate(eps.b):
        bc[i + 1] = bc[i + 1] - K * eps.wnorm * c
    op = 0
    for i, c in enumerate(bc):
        if c != 0.0:
            op = i
    return Sfilter(eps.wnorm, list(eps.b), bc[: op + 1])


def magnetic_susceptibility_impedance(mu: Sfilter, K: float) -> Sfilter:
    """Z(s)=s*K*(mu_r(s)-1), FILTER/filter_subroutines.F90:1309-1360."""
    aorder = len(mu.a) - 1 + 1
    ac = [0.0] * (aorder + 1)
    for i, c in enumerate(mu.a):
        ac[i + 1] = K * mu.wnorm * c
    for i, c in enumerate(mu.b):
        ac[i + 1] = ac[i + 1] - K * mu.wnorm * c
    op = 0
    for i, c in enumerate(ac):
        if c != 0.0:
            op = i
    return Sfilter(mu.wnorm, ac[: op + 1], list(mu.b))


@dataclass
class VolumeMaterial:
    """One entry of volume_material_list (TLM_material_modules.F90)."""

    type: int = MAT_DISPERSIVE
    eps: Sfilter = field(default_factory=lambda: Sfilter(1.0, [1.0], [1.0]))
    sigma_e: float = 0.0
    mu: Sfilter = field(default_factory=lambda: Sfilter(1.0, [1.0], [1.0]))
    sigma_m: float = 0.0

    @staticmethod
    def dielectric(eps_r: float, sigma: float = 0.0, mu_r: float = 1.0) -> "VolumeMaterial":
        return VolumeMaterial(MAT_DISPERSIVE, Sfilter(1.0, [eps_r], [1.0]), sigma, Sfilter(1.0, [mu_r], [1.0]), 0.0)

    @staticmethod
    def debye(eps_inf: float, delta_eps: Sequence[float], tau: Sequence[float], sigma: float = 0.0,
              wnorm: float = 1e9) -> "VolumeMaterial":
        """Multi-pole Debye eps(s)=eps_inf+sum d_i/(1+s tau_i) as a rational in
        s/wnorm (the .vmat format, e.g. TEST_DATA/MATERIAL_DATA/debye_1.vmat)."""
        den = [1.0]
        for t in tau:
            den = _poly_mul(den, [1.0, t * wnorm])
        num = [eps_inf * c for c in den]
        for i, (d, t) in enumerate(zip(delta_eps, tau)):
            other = [1.0]
            for j, t2 in enumerate(tau):
                if j != i:
                    other = _poly_mul(other, [1.0, t2 * wnorm])
            for k, c in enumerate(other):
                num[k] += d * c
        return VolumeMaterial(MAT_DISPERSIVE, Sfilter(wnorm, num, den), sigma, Sfilter(wnorm, [1.0], [1.0]), 0.0)


@dataclass
class SurfaceMaterial:
    """A dispersive thin layer (surface_material_type_DISPERSIVE or
    ANISOTROPIC_DISPERSIVE, TLM_MODULES/TLM_material_modules.F90): the
    S-domain two-port impedance filters ``z[pol][k]`` for the x, y and z
    polarisations (pol 0..2), k = 0..3 for Z11, Z12, Z21, Z22."""

    z: List[List[Sfilter]]


def surface_material_coefficients(sm: SurfaceMaterial, dt: float) -> dict:
    """calculate_surface_material_filter_coefficients
    (MATERIALS/TLM_surface_materials.F90:225-280): every filter through the
    bilinear transform and the fast/slow decomposition.  Returns f [3][4]
    (the fast parts), a, b [3][4][MAX_ORDER+1] (the slow Z filters, b(0)
    kept) and order [3][4]."""
    MO = MAX_ORDER + 1
    f = np.zeros((3, 4))
    a = np.zeros((3, 4, MO))
    b = np.zeros((3, 4, MO))
    order = np.zeros((3, 4), dtype=np.int32)
    for p in range(3):
        for k in range(4):
            za, zb = bilinear_s_to_z(sm.z[p][k], dt)
            ff, sa, sb = z_fast_slow_decomposition(za, zb)
            o = len(sb) - 1
            if o > MAX_ORDER:
                raise UnsupportedFeature(f"thin-layer filter of order {o} (at most {MAX_ORDER})")
            f[p, k] = ff
            a[p, k, :o + 1] = sa
            b[p, k, :o + 1] = sb
            order[p, k] = o
    return dict(f=f, a=a, b=b, order=order)


def material_coefficients(mat: VolumeMaterial, dl: float, dt: float, reduced_c: float = 1.0):
    """calculate_volume_material_filter_coefficients,
    MATERIALS/TLM_volume_materials.F90:190-385 (bilinear warp, frequency_scale=1)."""
    out = dict(type=mat.type, eps_exists=0, mu_exists=0, Ys_eps_f=0.0, Zs_mu_f=0.0, Ge=0.0, Rm=0.0,
               eps_a=[0.0], eps_b=[1.0], mu_a=[0.0], mu_b=[1.0], eps_order=0, mu_order=0)
    if mat.type != MAT_DISPERSIVE:
        return out
    Ge = mat.sigma_e * dl / reduced_c
    if Ge < 0.0:
        Ge = 0.0 if Ge >= -1e-12 else float("nan")
    out["Ge"] = Ge
    if not (len(mat.eps.a) == 1 and mat.eps.a[0] == 1.0):
        out["eps_exists"] = 1
        zs = electric_susceptibility_impedance(mat.eps, (EPS0 * reduced_c) * dl)
        a, b = bilinear_s_to_z(zs, dt)
        f_fast, a2, b2 = z_fast_slow_decomposition(a, b)
        out.update(Ys_eps_f=1.0 / f_fast, eps_a=a2, eps_b=b2, eps_order=max(len(a2), len(b2)) - 1)
    Rm = mat.sigma_m * dl
    if Rm < 0.0:
        Rm = 0.0 if Rm >= -1e-12 else float("nan")
    out["Rm"] = Rm
    if not (len(mat.mu.a) == 1 and mat.mu.a[0] == 1.0):
        out["mu_exists"] = 1
        zs = magnetic_susceptibility_impedance(mat.mu, (MU0 * reduced_c) * dl)
        a, b = bilinear_s_to_z(zs, dt)
        f_fast, a2, b2 = z_fast_slow_decomposition(a, b)
        out.update(Zs_mu_f=f_fast, mu_a=a2, mu_b=b2, mu_order=max(len(a2), len(b2)) - 1)
    return out


# ---------------------------------------------------------------------------
# Excitation functions (EXCITATION/excitation.F90:155-559)
# ---------------------------------------------------------------------------
@dataclass
class ExcitationFunction:
    """``type`` impulse | gaussian | gaussian_step | step | sinusoid |
    gaussian_sinusoid | differential_gaussian | gaussian_step_sinusoid |
    double_exponential | sinusoidal_pulse | ring_wave, or "file": a table of
    ``samples`` (times, values) read from a data file, evaluated as
    parameters[0] * interpolate_function(t - parameters[1])
    (EXCITATION/excitation.F90:522-540)."""

    type: str
    parameters: Tuple[float, ...]
    samples: Optional[Tuple[Sequence[float], Sequence[float]]] = None


def interpolate_function(time: float, times: Sequence[float], values: Sequence[float]) -> float:
    """EXCITATION/excitation.F90:710-768: the end values outside the table,
    else linear interpolation in the first interval [t_i, t_i+1] holding time."""
    if time <= times[0]:
        return float(values[0])
    if time >= times[-1]:
        return float(values[-1])
    for i in range(len(times) - 1):
        t1, t2 = times[i], times[i + 1]
        if t1 <= time <= t2:
            v1, v2 = values[i], values[i + 1]
            return float(v1 + (time - t1) * (v2 - v1) / (t2 - t1))
    raise ValueError(f"interpolate_function: no interval holds time {time!r}")


def excitation_tables(fns: Sequence[ExcitationFunction], n_timesteps: int, dt: float):
    """Tabulate value(t_n) and value_face(t_n+dt/2), excitation.F90:155-559.
    Scalar libm calls (math.exp / math.sin) so the tables are bitwise those of
    a glibc-linked build."""
    val = np.zeros((len(fns), n_timesteps))
    valf = np.zeros((len(fns), n_timesteps))
    for e, fn in enumerate(fns):
        p = fn.parameters
        for ts in range(1, n_timesteps + 1):
            time = (ts - 1) * dt
            time2 = time + dt / 2.0
            for k, t in ((0, time), (1, time2)):
                if fn.type == "impulse":
                    v = p[0] if ts == 1 else 0.0
                elif fn.type == "gaussian":
                    amp, width, delay = p[0], p[1], p[2]
                    v = amp * (math.exp(-(((t - delay) / width) ** 2))) if abs(t - delay) < width * 5.0 else 0.0
                elif fn.type == "gaussian_step":
                    amp, width, delay = p[0], p[1], p[2]
                    if t < delay:
                        v = amp * (math.exp(-(((t - delay) / width) ** 2))) if abs(t - delay) < width * 5.0 else 0.0
                    else:
                        v = amp
                elif fn.type == "step":
                    v = p[0] if t >= p[1] else 0.0
                elif fn.type == "sinusoid":
                    phase = p[2] * PI / 180.0
                    v = p[0] * math.sin(2.0 * PI * p[1] * t - phase)
                elif fn.type == "gaussian_sinusoid":
                    amp, width, delay, freq = p[0], p[1], p[2], p[3]
                    phase = p[4] * PI / 180.0
                    g = math.exp(-(((t - delay) / width) ** 2)) if abs(t - delay) < width * 5.0 else 0.0
                    v = amp * g * math.sin(2.0 * PI * freq * (t - delay) - phase)
                elif fn.type == "file":
                    if fn.samples is None or len(fn.samples[0]) < 1:
                        raise ValueError("a file excitation function without samples")
                    v = p[0] * interpolate_function(t - p[1], fn.samples[0], fn.samples[1])
                elif fn.type == "differential_gaussian":  # normalised to a peak of amplitude, :395-415
                    amp, width, delay = p[0], p[1], p[2]
                    tpeak = -width / math.sqrt(2.0)
                    fpeak = -2.0 * (tpeak / (width ** 2)) * math.exp(-((tpeak / width) ** 2))
                    if abs(t - delay) < width * 5.0:
                        v = -2.0 * ((t - delay) / width ** 2) * amp * math.exp(-(((t - delay) / width) ** 2)) / fpeak
                    else:
                        v = 0.0
                elif fn.type == "gaussian_step_sinusoid":  # :335-373
                    amp, width, delay, freq = p[0], p[1], p[2], p[3]
                    phase = p[4] * PI / 180.0
                    if t < delay:
                        g = math.exp(-(((t - delay) / width) ** 2)) if abs(t - delay) < width * 5 else 0.0
                    else:
                        g = 1.0
                    v = amp * g * math.sin(2.0 * PI * freq * t - phase)
                elif fn.type in ("double_exponential", "ring_wave"):  # :375-393, :485-513
                    # the face value takes 1/parameters(1) as its amplitude, as the reference does
                    amp = p[0] if k == 0 else 1.0 / p[0]
                    if t >= 0.0:
                        alpha, beta = 1.0 / p[1], 1.0 / p[2]
                        tpeak = (math.log(beta) - math.log(alpha)) / (beta - alpha)
                        fpeak = math.exp(-alpha * tpeak) - math.exp(-beta * tpeak)
                        v = (amp / fpeak) * (math.exp(-alpha * t) - math.exp(-beta * t))
                        if fn.type == "ring_wave":
                            v = v * math.sin(2.0 * PI * p[3] * t)
                    else:
                        v = 0.0
                elif fn.type == "sinusoidal_pulse":  # :448-483: trapezoidal envelope t1..t4
                    amp, freq, t1, t2, t3, t4 = p[0], p[1], p[3], p[4], p[5], p[6]
                    phase = p[2] * PI / 180.0
                    env = 0.0
                    if t1 <= t < t2:
                        env = (t - t1) / (t2 - t1)
                    elif t2 <= t <= t3:
                        env = 1.0
                    elif t3 <= t <= t4:
                        env = (t4 - t) / (t4 - t3)
                    v = amp * env * math.sin(2.0 * PI * freq * t - phase)
                else:
                    raise UnsupportedFeature(f"excitation function type {fn.type}")
                if k == 0:
                    val[e, ts - 1] = v
                else:
                    valf[e, ts - 1] = v
    return val, valf


# ---------------------------------------------------------------------------
# Problem specification (the .inp + .mesh content this path consumes)
# ---------------------------------------------------------------------------
@dataclass
class Block:
    """Axis-aligned block of cells, 1-based inclusive cell ranges."""

    i0: int
    i1: int
    j0: int
    j1: int
    k0: int
    k1: int


@dataclass
class CellList:
    """An explicit set of cells (1-based i, j, k rows): a volume as the
    reference's mesher voxelised it, read from a mesh file's cell list
    (MESH/read_mesh.F90:112-160)."""

    cells: np.ndarray

    def __post_init__(self):
        self.cells = np.asarray(self.cells, dtype=np.int64).reshape(-1, 3)


@dataclass
class Sphere:
    """Cells whose centres lie inside a sphere (centre and radius in cells,
    cell centres at integer+0.5 in 0-based cell coordinates)."""

    cx: float
    cy: float
    cz: float
    r: float


@dataclass
class PointExcitation:
    cell: Tuple[int, int, int]  # 1-based
    component: str
    function: int  # 1-based function number
    source_type: int = SOURCE_SOFT
    face: str = "centre"  # or xmin, xmax, ymin, ymax, zmin, zmax: a point source on that face of the cell
    # a face source on that side of the face alone (side 1 for a min face, 2 for a max face), as
    # Surface_excitation applies a one-sided surface (excitation_surfaces.F90:236-262); a point
    # source on a face reaches both sides (excitation_points.F90:286-323)
    one_side: bool = False
    # the function's value times this factor: a mode excitation's mode field, halved when it
    # excites both sides (mode_excitation.F90:393-411)
    scale: float = 1.0


@dataclass
class HuygensPlane:
    """A planar Huygens patch on cell faces.  ``axis`` 1..3 is the face
    normal; the patch lies on the boundary between cells ``index`` and
    ``index+1`` along that axis and covers the 1-based inclusive transverse
    cell ranges ``r0``, ``r1``.  ``side`` is the side flag of the
    Huygens_surface packet (1 or -1).  For a planar rectangle the reference's
    surface mesher records each face as the min face of the cell on the +axis
    side (outward normal -axis); side 1 keeps that face, side -1 moves the
    excitation to the max face of the cell below (huygens_surface.F90:420-460).
    This convention is pinned by TEST_DATA/TEM_PML_TEST Ey.tout_ref, where a
    +z plane wave launched from such a patch with side 1 reproduces the golden
    series.  Angles in degrees as in the .inp packet."""

    axis: int
    index: int
    r0: Tuple[int, int]
    r1: Tuple[int, int]
    function: int
    ktheta: float
    kphi: float
    etheta: float
    ephi: float
    side: int = 1
    wave_impedance: float = Z0  # the optional wave_impedance line (read_huygens_surface.F90:107-116)


@dataclass
class HuygensBox:
    """A closed Huygens surface on the boundary faces of the block of cells
    i0..i1, j0..j1, k0..k1 (1-based, inclusive): the reference's
    rectangular_block surface aligned with the mesh.  Its triangles
    (GEOMETRY/build_surface_rectangular_block.F90) have normals that point
    into the block under triangle_normal's (v3-v1)x(v2-v1)
    (GEOMETRY/functions.F90:241-262), and the surface mesher
    (MESH/mesh_triangle.F90) records each face on the cell behind the
    triangle, facing along that normal: with side 1 the patches sit on the
    neighbouring outside cells with inward normals, and the incident field
    appears inside the block.  Side -1 moves every patch to the block's own
    boundary cell with an outward normal.  Pinned by TEST_DATA/HUYGENS_SURFACE
    (*_centre.tout_ref)."""

    i: Tuple[int, int]
    j: Tuple[int, int]
    k: Tuple[int, int]
    function: int
    ktheta: float
    kphi: float
    etheta: float
    ephi: float
    side: int = 1
    wave_impedance: float = Z0  # the optional wave_impedance line (read_huygens_surface.F90:107-116)


@dataclass
class HuygensOuter:
    """The Huygens surface on the outer boundary of the mesh (surface number
    0 in the Huygens_surface packet, huygens_surface%outer_surface_flag):
    every boundary face is a patch with the outward normal of the mesh
    (huygens_surface.F90:517-612), and its J, M enter the boundary ports in
    outer_boundary (TLM_SOLVER/outer_boundary.F90:133-318)."""

    function: int
    ktheta: float
    kphi: float
    etheta: float
    ephi: float
    wave_impedance: float = Z0


@dataclass
class FarFieldSurface:
    """A far-field surface (Far_field_surface packet, OUTPUT/far_field_surfaces.F90):
    per frequency the accumulators J += e^{-jwt} dt (n x H) and
    M -= e^{-jwt} dt (n x E) of every face of a closed box of cells
    ``box`` = ((i0, i1), (j0, j1), (k0, k1)) or of a planar patch ``plane`` =
    (axis, index, r0, r1).  The faces are those the surface mesher records
    (as for HuygensBox / HuygensPlane), flipped to the other side of each
    face when ``side`` is -1; n is +1 on a min face and -1 on a max face,
    i.e. it points into the cell whose face is sampled."""

    frequencies: List[float]
    box: Optional[Tuple[Tuple[int, int], Tuple[int, int], Tuple[int, int]]] = None
    plane: Optional[Tuple[int, int, Tuple[int, int], Tuple[int, int]]] = None
    side: int = 1
    # or the surface's faces as a mesh file lists them: (cell, face code) per
    # face before the side flip (MESH/read_mesh.F90:186-225)
    records: Optional[List[Tuple[Tuple[int, int, int], int]]] = None

    def faces(self) -> List[Tuple[Tuple[int, int, int], int]]:
        if sum(g is not None for g in (self.box, self.plane, self.records)) != 1:
            raise ValueError("a far-field surface is a box, a plane or a list of mesh faces")
        if self.records is not None:
            return _side_flip(self.records, self.side)
        if self.box is not None:
            g = HuygensBox(self.box[0], self.box[1], self.box[2], 0, 0.0, 0.0, 1.0, 0.0, side=self.side)
        else:
            ax, ix, r0, r1 = self.plane
            g = HuygensPlane(ax, ix, r0, r1, 0, 0.0, 0.0, 1.0, 0.0, side=self.side)
        return _huygens_patches(g)


# output surface components: E, H, J = n x H, and the magnitudes
# |E|, |H|, |J| (TLM_MODULES/TLM_Modules.F90:178-180)
SURFACE_COMPONENTS = {"Ex": 1, "Ey": 2, "Ez": 3, "Hx": 4, "Hy": 5, "Hz": 6, "Jx": 7, "Jy": 8, "Jz": 9,
                      "Em": 13, "Hm": 14, "Jm": 15}


@dataclass
class OutputSurface:
    """A time-domain output surface (Output_surface packet,
    OUTPUT/output_surfaces.F90): on the output steps first..last every
    ``interval`` (last None = the final step), the value of ``component``
    (SURFACE_COMPONENTS) on every face of a closed box of cells ``box`` or a
    planar patch ``plane``, faces as for FarFieldSurface (``side`` -1 samples
    the other side of each face, output_on_outward_normal false).  With
    ``both_sides`` (output_average_of_both_sides) J is n x H of side 1 minus
    n x H of side 2; other components read side 1."""

    component: str
    box: Optional[Tuple[Tuple[int, int], Tuple[int, int], Tuple[int, int]]] = None
    plane: Optional[Tuple[int, int, Tuple[int, int], Tuple[int, int]]] = None
    side: int = 1
    both_sides: bool = False
    first_step: int = 1
    last_step: Optional[int] = None
    interval: int = 1
    records: Optional[List[Tuple[Tuple[int, int, int], int]]] = None  # mesh faces, as for FarFieldSurface

    def faces(self) -> List[Tuple[Tuple[int, int, int], int]]:
        return FarFieldSurface([], self.box, self.plane, self.side, self.records).faces()


@dataclass
class RCSSurface:
    """The RCS surface (RCS_surface packet, OUTPUT/RCS_surfaces.F90): the
    faces of a closed box or planar patch as for FarFieldSurface, and the
    far-field direction ``theta``, ``phi`` in degrees
    (read_rcs_surface.F90:79-86 turns them into radians)."""

    theta: float
    phi: float
    box: Optional[Tuple[Tuple[int, int], Tuple[int, int], Tuple[int, int]]] = None
    plane: Optional[Tuple[int, int, Tuple[int, int], Tuple[int, int]]] = None
    side: int = 1
    records: Optional[List[Tuple[Tuple[int, int, int], int]]] = None  # mesh faces, as for FarFieldSurface

    def faces(self) -> List[Tuple[Tuple[int, int, int], int]]:
        return FarFieldSurface([], self.box, self.plane, self.side, self.records).faces()


RCS_POINTS_PER_CELL = 2  # n_rcs_points_per_cell, TLM_MODULES/TLM_output_modules.F90:388

# surface_material_type_*, TLM_MODULES/TLM_material_modules.F90:153-161; a
# dispersive and an anisotropic dispersive layer take the same update
SURFACE_SHEET_TYPES = {"PEC": 1, "PMC": 2, "dispersive": 3, "free": 4}


@dataclass
class SurfaceSheet:
    """A PEC, PMC or free-space surface material on a planar patch of
    internal cell faces (the same (axis, index, r0, r1) convention as
    DFTSurface): the connect across those faces reflects each side with -1
    (PEC) or +1 (PMC), or is the plain connect (free space)
    (connect_normal_to_x.F90:36-52).  Thin-layer and other surface
    materials stay unsupported."""

    kind: str
    axis: int
    index: int
    r0: Tuple[int, int]
    r1: Tuple[int, int]
    # explicit faces instead of the patch: ((cx, cy, cz) of the cell on the
    # + side, axis) per face, e.g. a triangulated surface as the reference's
    # mesher put it on cell faces (read from a mesh file)
    faces: Optional[List[Tuple[Tuple[int, int, int], int]]] = None
    # a "dispersive" sheet: its thin-layer material (1-based into
    # ProblemSpec.thin_layers) and, per face (or one value for all), the
    # sign set_surface_material_mesh (TLM_surface_materials.F90:150-175)
    # gives the face's min-face entry: the orientation list's sign, negated
    # where the surface records the max face of the cell below.  The
    # connect treats the layer as reversed where the sign is positive
    # (connect_normal_to_x.F90:14-19).
    material: int = 0
    sign: object = 1

    def face_keys(self):
        if self.faces is not None:
            return list(self.faces)
        return [(f, self.axis) for f in _plane_faces(self.axis, self.index, self.r0, self.r1)]

    def face_signs(self) -> List[int]:
        n = len(self.face_keys())
        return [int(v) for v in self.sign] if isinstance(self.sign, (list, tuple)) else [int(self.sign)] * n


@dataclass
class PowerSurface:
    """A frequency-domain power surface (OUTPUT/frequency_domain_power_surfaces.F90):
    faces of a box or plane as for FarFieldSurface and a list of
    frequencies; every step each face accumulates the DFT of the two
    tangential E and H components on its side."""

    frequencies: Sequence[float]
    box: Optional[Tuple[Tuple[int, int], Tuple[int, int], Tuple[int, int]]] = None
    plane: Optional[Tuple[int, int, Tuple[int, int], Tuple[int, int]]] = None
    side: int = 1
    records: Optional[List[Tuple[Tuple[int, int, int], int]]] = None  # mesh faces, as for FarFieldSurface

    def faces(self) -> List[Tuple[Tuple[int, int, int], int]]:
        return FarFieldSurface([], self.box, self.plane, self.side, self.records).faces()


@dataclass
class ModeOutput:
    """A mode output (OUTPUT/output_modes.F90): every step the sum over the
    faces of a plane patch of one field component on each face's side
    times the mode field ``profile(i, j, k)`` of the face's cell, or over
    ``samples`` (cell, face code, mode field) in their order, as the reader
    takes them from a mode file (set_mode_outputs_in_mesh)."""

    component: str
    plane: Optional[Tuple[int, int, Tuple[int, int], Tuple[int, int]]]
    profile: object
    side: int = 1
    samples: Optional[List[Tuple[Tuple[int, int, int], int, float]]] = None

    def faces(self) -> List[Tuple[Tuple[int, int, int], int]]:
        if self.samples is not None:
            return [(tuple(int(v) for v in c), int(code)) for c, code, _ in self.samples]
        return FarFieldSurface([], None, self.plane, self.side).faces()

    def weights(self) -> List[float]:
        if self.samples is not None:
            return [float(w) for _, _, w in self.samples]
        return [float(self.profile(*c)) for c, _ in self.faces()]


@dataclass
class OutputPoint:
    cell: Tuple[int, int, int]
    component: str
    face: str = "centre"  # or a face of the cell (field on that side of the face, after connect)


@dataclass
class DFTSurface:
    """Frequency-domain output surface: a planar face patch (same convention
    as HuygensPlane) and a list of frequencies for one field component.
    ``records`` (a mesh file's faces, as for FarFieldSurface) replace the
    patch; ``side`` -1 samples the other side of each face."""

    axis: int
    index: int
    r0: Tuple[int, int]
    r1: Tuple[int, int]
    frequencies: Sequence[float]
    component: str
    side: int = 1
    records: Optional[List[Tuple[Tuple[int, int, int], int]]] = None
    first_step: int = 1            # output steps first..last every interval
    last_step: Optional[int] = None  # (get_output_flag, output.F90:564-598); None = the final step
    interval: int = 1

    def faces(self) -> List[Tuple[Tuple[int, int, int], int]]:
        if self.records is not None:
            return _side_flip(self.records, self.side)
        return _side_flip([(c, self.axis) for c in _plane_faces(self.axis, self.index, self.r0, self.r1)],
                          self.side)


@dataclass
class FrequencyOutputVolume:
    """Frequency-domain output volume (OUTPUT/frequency_output_volumes.F90):
    the cells of a region (Block or Sphere), optionally only every
    ``every``-th cell per axis counted from the region's lowest cell
    (frequency_output_volume_output_every, :58-108), one field component
    Ex..Hz, a list of frequencies, and the output steps first..last every
    ``interval`` (output.F90:564-598; last None = the final step)."""

    region: object
    frequencies: Sequence[float]
    component: str
    first_step: int = 1
    last_step: Optional[int] = None
    interval: int = 1
    every: int = 1

    def mask(self, spec: "ProblemSpec") -> np.ndarray:
        m = _region_mask(spec, self.region)
        if self.every > 1 and m.any():
            z, y, x = np.nonzero(m)
            keep = (((x - x.min()) % self.every == 0) & ((y - y.min()) % self.every == 0) &
                    ((z - z.min()) % self.every == 0))
            m = np.zeros_like(m)
            m[z[keep], y[keep], x[keep]] = True
        return m


OUTPUT_VOLUME_KINDS = {"field": 0, "average": 1, "peak": 2}


@dataclass
class SARVolume:
    """A SAR volume (SAR_volume packet, OUTPUT/SAR_volumes.F90): the cells of
    a region, optionally every ``every``-th per axis, and a list of
    frequencies; every step each cell accumulates the DFT of Ex, Ey, Ez
    times dt, from which write_SAR_volumes computes SAR on the host."""

    region: object
    frequencies: Sequence[float]
    every: int = 1

    def mask(self, spec: "ProblemSpec") -> np.ndarray:
        return FrequencyOutputVolume(self.region, [], "Ex", every=self.every).mask(spec)


@dataclass
class OutputVolume:
    """A time-domain output volume on the output steps first..last every
    ``interval``: ``kind`` "field" records each cell's ``component``
    (OUTPUT/output_volumes.F90), "average" their mean
    (output_volume_averages.F90), "peak" the largest magnitude
    (output_volume_peak.F90).  Cells as for FrequencyOutputVolume."""

    region: object
    component: str
    kind: str = "field"
    first_step: int = 1
    last_step: Optional[int] = None
    interval: int = 1
    every: int = 1

    def mask(self, spec: "ProblemSpec") -> np.ndarray:
        return FrequencyOutputVolume(self.region, [], self.component, every=self.every).mask(spec)


@dataclass
class ProblemSpec:
    nx: int
    ny: int
    nz: int
    dl: float
    n_timesteps: int
    R: Tuple[float, float, float, float, float, float] = (0.0,) * 6
    # Wrapping_boundary_conditions (read_wrapping_boundary_conditions.F90):
    # 1 joins the two outer faces of that axis (wrap_outer_boundary.F90)
    wrap: Tuple[int, int, int] = (0, 0, 0)
    origin: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    pml_cells: Tuple[int, int, int, int, int, int] = (0,) * 6
    pml_r: Tuple[float, ...] = (1e-4,) * 6
    pml_order: int = 2
    materials: List[VolumeMaterial] = field(default_factory=list)
    material_regions: List[Tuple[int, object]] = field(default_factory=list)  # (material number, Block|Sphere)
    functions: List[ExcitationFunction] = field(default_factory=list)
    point_excitations: List[PointExcitation] = field(default_factory=list)
    huygens: Optional[object] = None  # HuygensPlane, HuygensBox or HuygensOuter
    outputs: List[OutputPoint] = field(default_factory=list)
    dft_surfaces: List[DFTSurface] = field(default_factory=list)
    far_field_surfaces: List["FarFieldSurface"] = field(default_factory=list)
    frequency_output_volumes: List[FrequencyOutputVolume] = field(default_factory=list)
    output_surfaces: List[OutputSurface] = field(default_factory=list)
    surface_sheets: List[SurfaceSheet] = field(default_factory=list)
    thin_layers: List[SurfaceMaterial] = field(default_factory=list)  # materials of the "dispersive" sheets
    rcs_surface: Optional[RCSSurface] = None
    power_surfaces: List[PowerSurface] = field(default_factory=list)
    mode_outputs: List[ModeOutput] = field(default_factory=list)
    output_volumes: List[OutputVolume] = field(default_factory=list)
    sar_volumes: List[SARVolume] = field(default_factory=list)
    reduced_c: float = 1.0
    # the Simulation_time packet's value (read_simulation_time), where the
    # problem came from a problem file; n_timesteps = NINT(simulation_time/dt)
    simulation_time: Optional[float] = None
    # set_small_to_zero packet (read_small_to_zero.F90:55-59): (n_small_to_zero, small_to_zero_value)
    small_to_zero: Optional[Tuple[int, float]] = None
    # features rejected up front by the GPU path
    cables: int = 0
    ngspice: bool = False
    surface_materials: int = 0


def _region_mask(spec: ProblemSpec, region) -> np.ndarray:
    """Boolean [nz, ny, nx] mask of the cells of a region."""
    m = np.zeros((spec.nz, spec.ny, spec.nx), dtype=bool)
    if isinstance(region, Block):
        m[region.k0 - 1:region.k1, region.j0 - 1:region.j1, region.i0 - 1:region.i1] = True
    elif isinstance(region, Sphere):
        lo = [max(0, int(math.floor(c - region.r)) - 1) for c in (region.cz, region.cy, region.cx)]
        hi = [min(n, int(math.ceil(c + region.r)) + 1) for c, n in
              ((region.cz, spec.nz), (region.cy, spec.ny), (region.cx, spec.nx))]
        z, y, x = np.meshgrid(np.arange(lo[0], hi[0]) + 0.5, np.arange(lo[1], hi[1]) + 0.5,
                              np.arange(lo[2], hi[2]) + 0.5, indexing="ij")
        m[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = (
            (x - region.cx) ** 2 + (y - region.cy) ** 2 + (z - region.cz) ** 2 <= region.r ** 2)
    elif isinstance(region, CellList):
        c = region.cells
        if c.size:
            if (c.min(axis=0) < 1).any() or (c.max(axis=0) > (spec.nx, spec.ny, spec.nz)).any():
                raise ValueError("a cell list reaches outside the mesh")
            m[c[:, 2] - 1, c[:, 1] - 1, c[:, 0] - 1] = True
    else:
        raise TypeError(region)
    return m


def _plane_faces(axis: int, index: int, r0, r1):
    """Cell faces of a planar patch: list of (cx,cy,cz) of the cell on the +
    side of each face (the cell whose *min* face it is), in connect order."""
    faces = []
    if axis == 1:
        for k in range(r1[0], r1[1] + 1):
            for j in range(r0[0], r0[1] + 1):
                faces.append((index + 1, j, k))
    elif axis == 2:
        for k in range(r1[0], r1[1] + 1):
            for i in range(r0[0], r0[1] + 1):
                faces.append((i, index + 1, k))
    else:
        for j in range(r1[0], r1[1] + 1):
            for i in range(r0[0], r0[1] + 1):
                faces.append((i, j, index + 1))
    return faces


def calc_pml_dist(c: int, n: int, t_min: int, t_max: int) -> Tuple[int, int]:
    """MATERIALS/TLM_PML_volume_materials.F90:446-481."""
    d_min = c
    d_max = n - c + 1
    dist_min = d_min - (t_min + 1)
    if dist_min > 0:
        dist_min = 0
    dist_max = t_max - d_max + 1
    if dist_max < 0:
        dist_max = 0
    return dist_min, dist_max


def calc_sigma_0(r: float, N: int, order: int, dl: float) -> float:
    """MATERIALS/TLM_PML_volume_materials.F90:498-513."""
    if N == 0:
        return float("inf")
    return -(EPS0 * C0 / 2.0) * math.log(r) / (dl * float(abs(N) ** (order + 1)))


def pml_conductivity(d: int, n_min: int, n_max: int, s0_min: float, s0_max: float, order: int) -> float:
    """MATERIALS/TLM_PML_volume_materials.F90:531-581."""
    if d == 0:
        return 0.0
    L = abs(d) - 1
    s0 = s0_min if d < 0 else s0_max
    return s0 * float((L + 1) ** (order + 1) - L ** (order + 1))


def pml_parameter_row(sx: float, sy: float, sz: float, dt: float) -> List[float]:
    """One PML_parameters row, TLM_PML_volume_materials.F90:333-351."""
    return [
        4.0 / (4.0 + (sy + sz) * dt), 4.0 / (4.0 + (sz + sx) * dt), 4.0 / (4.0 + (sx + sy) * dt),
        math.exp(-dt * sx / 2.0), math.exp(-dt * sy / 2.0), math.exp(-dt * sz / 2.0),
        sx * dt / 4.0, sy * dt / 4.0, sz * dt / 4.0,
        sx * dt / 2.0, sy * dt / 2.0, sz * dt / 2.0,
        1.0 - (sy + sz) * dt / 4.0, 1.0 - (sz + sx) * dt / 4.0, 1.0 - (sx + sy) * dt / 4.0,
    ]


def huygens_vectors(ktheta_deg: float, kphi_deg: float, etheta: float, ephi: float, hs_z0: float = Z0):
    """K, Ei, Hi of set_huygens_surface_data, EXCITATION/huygens_surface.F90:300-360."""
    theta = (PI / 180.0) * ktheta_deg
    phi = (PI / 180.0) * kphi_deg
    r = 1.0
    # rthetaphi_to_xyz_point
    kx = r * math.sin(theta) * math.cos(phi)
    ky = r * math.sin(theta) * math.sin(phi)
    kz = r * math.cos(theta)
    dxdt = r * math.cos(theta) * math.cos(phi)
    dxdp = -r * math.sin(phi)
    dydt = r * math.cos(theta) * math.sin(phi)
    dydp = r * math.cos(phi)
    dzdt = -r * math.sin(theta)
    dzdp = 0.0
    vx = etheta * dxdt + ephi * dxdp
    vy = etheta * dydt + ephi * dydp
    vz = etheta * dzdt + ephi * dzdp
    norm = math.sqrt(vx * vx + vy * vy + vz * vz)
    Ei = [vx / norm, vy / norm, vz / norm]
    Hi = [ky * Ei[2] - kz * Ei[1], kz * Ei[0] - kx * Ei[2], kx * Ei[1] - ky * Ei[0]]
    Hi = [h / hs_z0 for h in Hi]
    return (kx, ky, kz), Ei, Hi


def _huygens_patches(hs) -> List[Tuple[Tuple[int, int, int], int]]:
    """(cell, face code 1..6) of every Huygens patch after the side flip
    (huygens_surface.F90:412-450), in the surface mesher's face_list order
    (face code, then cz, cy, cx; MESH/build_surface_mesh.F90:100-150)."""
    rec = []
    if isinstance(hs, HuygensOuter):
        raise TypeError("the outer-boundary surface has no connect faces")
    if isinstance(hs, HuygensPlane):
        # recorded as the min face of the cell on the + side (normal -axis)
        for c in _plane_faces(hs.axis, hs.index, hs.r0, hs.r1):
            rec.append((c, hs.axis))
    else:
        (i0, i1), (j0, j1), (k0, k1) = hs.i, hs.j, hs.k
        if i0 > i1 or j0 > j1 or k0 > k1:
            raise ValueError("empty Huygens box")
        # min faces of the cells just past the block's max planes, max faces
        # of the cells just before its min planes (inward normals)
        for code in (FACE_XMIN, FACE_YMIN, FACE_ZMIN, FACE_XMAX, FACE_YMAX, FACE_ZMAX):
            axis = (code - 1) % 3
            at = (i1 + 1, j1 + 1, k1 + 1)[axis] if code <= 3 else (i0 - 1, j0 - 1, k0 - 1)[axis]
            rng = [range(i0, i1 + 1), range(j0, j1 + 1), range(k0, k1 + 1)]
            rng[axis] = range(at, at + 1)
            for cz in rng[2]:
                for cy in rng[1]:
                    for cx in rng[0]:
                        rec.append(((cx, cy, cz), code))
    return _side_flip(rec, hs.side)


def _side_flip(rec, side: int) -> List[Tuple[Tuple[int, int, int], int]]:
    """(cell, face code) records as they are, for side 1, or each moved to
    the same face seen from the neighbouring cell, for side -1
    (huygens_surface.F90:412-450 and the output surfaces' side flag)."""
    out = []
    for c, code in rec:
        c = tuple(int(v) for v in c)
        if side != 1:
            axis = (code - 1) % 3
            c = list(c)
            c[axis] += -1 if code <= 3 else 1
            code = code + 3 if code <= 3 else code - 3
            c = tuple(c)
        out.append((c, int(code)))
    return out


def build_tables(spec: ProblemSpec) -> dict:
    """Produce the full table set for one problem (everything the C-ABI
    ``tlm_gpu_set_*`` entry points and the oracle consume)."""
    if spec.cables:
        raise UnsupportedFeature("cable models are not supported by the GPU path")
    if spec.ngspice:
        raise UnsupportedFeature("Ngspice co-simulation is not supported by the GPU path")
    if spec.surface_materials:
        raise UnsupportedFeature("surface (thin-layer) materials are not supported by the GPU path")
    nx, ny, nz, dl = spec.nx, spec.ny, spec.nz, spec.dl
    dt = dl / (2.0 * C0 / spec.reduced_c)  # set_TLM_solver_parameters.F90:94
    nsteps = spec.n_timesteps
    ncell = nx * ny * nz

    # local_cell_material / local_cell_PML / local_cell_excitation / local_cell_output
    cell_mat = np.zeros((nz, ny, nx), dtype=np.int32)
    for mnum, region in spec.material_regions:
        cell_mat[_region_mask(spec, region)] = mnum
    t = spec.pml_cells
    dxa = np.zeros(nx, dtype=np.int32)
    dya = np.zeros(ny, dtype=np.int32)
    dza = np.zeros(nz, dtype=np.int32)
    for arr, n, tmin, tmax in ((dxa, nx, t[0], t[1]), (dya, ny, t[2], t[3]), (dza, nz, t[4], t[5])):
        for c in range(1, n + 1):
            dmin, dmax = calc_pml_dist(c, n, tmin, tmax)
            arr[c - 1] = dmin if dmin != 0 else dmax
    in_pml = (dza[:, None, None] != 0) | (dya[None, :, None] != 0) | (dxa[None, None, :] != 0)
    for q in list(spec.point_excitations) + list(spec.outputs):
        if q.face != "centre" and q.face not in FACE_POINT:
            raise ValueError(f"unknown face {q.face!r}")
    centre_pts = [q for q in spec.point_excitations if q.face == "centre"]
    if any(q.scale != 1.0 or q.one_side for q in centre_pts):
        raise ValueError("a centre point excitation takes neither a scale nor a side")
    centre_outs = [q for q in spec.outputs if q.face == "centre"]
    cell_exc = np.zeros((nz, ny, nx), dtype=bool)
    for pe in centre_pts:
        if COMPONENTS[pe.component] > 9:
            raise ValueError("a cell-centre source drives E, H or J (components 1..9)")
        i, j, k = pe.cell
        cell_exc[k - 1, j - 1, i - 1] = True
    cell_out = np.zeros((nz, ny, nx), dtype=bool)
    for op in centre_outs:
        i, j, k = op.cell
        cell_out[k - 1, j - 1, i - 1] = True
    point_out = cell_out.copy()  # output points keep a time series; volume cells need only the current step
    vol_masks = []
    for fv in spec.frequency_output_volumes:
        if COMPONENTS.get(fv.component, 0) not in range(1, 7):
            raise ValueError("a frequency output volume records Ex..Hz")
        if fv.interval < 1 or fv.every < 1:
            raise ValueError("frequency output volume interval and cell spacing must be >= 1")
        vm = fv.mask(spec)
        vol_masks.append(vm)
        cell_out |= vm
    sar_masks = []
    for sv in spec.sar_volumes:
        if sv.every < 1:
            raise ValueError("SAR volume cell spacing must be >= 1")
        vm = sv.mask(spec)
        sar_masks.append(vm)
        cell_out |= vm
    ovol_masks = []
    for ov in spec.output_volumes:
        if COMPONENTS.get(ov.component, 0) not in range(1, 7):
            raise ValueError("an output volume records Ex..Hz")
        if ov.kind not in OUTPUT_VOLUME_KINDS or ov.first_step < 1 or ov.interval < 1 or ov.every < 1:
            raise ValueError("output volume kind, first step, interval or cell spacing")
        vm = ov.mask(spec)
        ovol_masks.append(vm)
        cell_out |= vm
    if np.any(in_pml & cell_exc):
        raise UnsupportedFeature("Excitation intersects PML")  # set_update_codes.F90:347-354
    special = (cell_mat != 0) | in_pml | cell_exc | cell_out
    # materials in the PML (set_update_codes.F90:290-331, scatter.F90:552-567):
    # PEC/PMC stop the reference, so do dispersive ones (any S-domain order
    # above 0); a constant eps_r, mu_r, sigma material takes the PML-material
    # update (scatter_PML_material.F90)
    for mnum in np.unique(cell_mat[in_pml & (cell_mat != 0)]):
        vm = spec.materials[int(mnum) - 1]
        if vm.type != MAT_DISPERSIVE:
            raise UnsupportedFeature("PEC/PMC volume material in PML")
        if len(vm.eps.a) > 1 or len(vm.eps.b) > 1 or len(vm.mu.a) > 1 or len(vm.mu.b) > 1:
            raise UnsupportedFeature(f"PML fatal error: dispersive material found, material number {int(mnum)}")

    # set_cell_update_codes, set_update_codes.F90:38-363 (traversal order cz,cy,cx)
    flat_special = special.reshape(-1)
    n_special = int(flat_special.sum())
    cell_code = np.zeros(ncell, dtype=np.int32)
    cell_code[flat_special] = np.arange(1, n_special + 1, dtype=np.int32)
    sp_material = cell_mat.reshape(-1)[flat_special].astype(np.int32)
    exc_flat = cell_exc.reshape(-1)[flat_special]
    out_flat = cell_out.reshape(-1)[flat_special]
    sp_excitation = exc_flat.astype(np.int32)
    sp_output = out_flat.astype(np.int32)
    # excitation / output cell numbers in traversal order
    exc_number = np.zeros(ncell, dtype=np.int32)
    exc_number[cell_exc.reshape(-1)] = np.arange(1, int(cell_exc.sum()) + 1)
    out_number = np.zeros(ncell, dtype=np.int32)
    out_number[cell_out.reshape(-1)] = np.arange(1, int(cell_out.sum()) + 1)

    # PML cell numbering and parameter table, TLM_PML_volume_materials.F90:41-428
    pml_flat = in_pml.reshape(-1)
    n_pml = int(pml_flat.sum())
    pml_number = np.zeros(ncell, dtype=np.int32)
    pml_number[pml_flat] = np.arange(1, n_pml + 1, dtype=np.int32)
    sp_pml = pml_number[flat_special].astype(np.int32)
    pml_params = np.zeros((0, 15))
    pml_sigma = np.zeros((0, 3))
    pml_cell_param = np.zeros(0, dtype=np.int32)
    if n_pml:
        zz, yy, xx = np.nonzero(in_pml)
        dx_c, dy_c, dz_c = dxa[xx], dya[yy], dza[zz]
        pml_xmin, pml_xmax = min(0, int(dx_c.min())), max(0, int(dx_c.max()))
        pml_ymin, pml_ymax = min(0, int(dy_c.min())), max(0, int(dy_c.max()))
        pml_zmin, pml_zmax = min(0, int(dz_c.min())), max(0, int(dz_c.max()))
        o = spec.pml_order
        r = spec.pml_r
        s0 = [calc_sigma_0(r[0], pml_xmin, o, dl) / EPS0, calc_sigma_0(r[1], pml_xmax, o, dl) / EPS0,
              calc_sigma_0(r[2], pml_ymin, o, dl) / EPS0, calc_sigma_0(r[3], pml_ymax, o, dl) / EPS0,
              calc_sigma_0(r[4], pml_zmin, o, dl) / EPS0, calc_sigma_0(r[5], pml_zmax, o, dl) / EPS0]
        keys = np.stack([dx_c, dy_c, dz_c], axis=1)
        uniq, first_idx, inverse = np.unique(keys, axis=0, return_index=True, return_inverse=True)
        order = np.argsort(first_idx)  # parameters numbered in first-seen traversal order
        rank = np.empty_like(order)
        rank[order] = np.arange(len(order))
        pml_cell_param = (rank[inverse.reshape(-1)] + 1).astype(np.int32)
        pml_params = np.zeros((len(uniq), 15))
        pml_sigma = np.zeros((len(uniq), 3))
        for u in range(len(uniq)):
            ddx, ddy, ddz = (int(v) for v in uniq[u])
            sx = pml_conductivity(ddx, pml_xmin, pml_xmax, s0[0], s0[1], o)
            sy = pml_conductivity(ddy, pml_ymin, pml_ymax, s0[2], s0[3], o)
            sz = pml_conductivity(ddz, pml_zmin, pml_zmax, s0[4], s0[5], o)
            pml_params[rank[u]] = pml_parameter_row(sx, sy, sz, dt)
            pml_sigma[rank[u]] = (sx, sy, sz)

    # volume materials
    mats = [material_coefficients(m, dl, dt, spec.reduced_c) for m in spec.materials]
    nm = len(mats)
    MO = MAX_ORDER + 1

    def coef(key):
        arr = np.zeros((max(nm, 1), MO))
        for i, m in enumerate(mats):
            c = m[key]
            arr[i, : len(c)] = c
        return arr

    tables = dict(
        nx=nx, ny=ny, nz=nz, dl=dl, dt=dt, n_timesteps=nsteps, R=np.array(spec.R, dtype=np.float64),
        cell_code=cell_code, n_special=n_special, sp_material=sp_material, sp_pml=sp_pml,
        sp_excitation=sp_excitation, sp_output=sp_output,
        n_materials=nm,
        mat_type=np.array([m["type"] for m in mats] or [0], dtype=np.int32),
        mat_eps_exists=np.array([m["eps_exists"] for m in mats] or [0], dtype=np.int32),
        mat_mu_exists=np.array([m["mu_exists"] for m in mats] or [0], dtype=np.int32),
        mat_eps_order=np.array([m["eps_order"] for m in mats] or [0], dtype=np.int32),
        mat_mu_order=np.array([m["mu_order"] for m in mats] or [0], dtype=np.int32),
        mat_Ys_eps_f=np.array([m["Ys_eps_f"] for m in mats] or [0.0]),
        mat_Zs_mu_f=np.array([m["Zs_mu_f"] for m in mats] or [0.0]),
        mat_Ge=np.array([m["Ge"] for m in mats] or [0.0]),
        mat_Rm=np.array([m["Rm"] for m in mats] or [0.0]),
        mat_eps_a=coef("eps_a"), mat_eps_b=coef("eps_b"), mat_mu_a=coef("mu_a"), mat_mu_b=coef("mu_b"),
        n_pml_params=len(pml_params), pml_params=np.ascontiguousarray(pml_params, dtype=np.float64),
        n_pml_cells=n_pml, pml_cell_param=pml_cell_param,
        pml_sigma=np.ascontiguousarray(pml_sigma, dtype=np.float64),
        n_pml_material_cells=int(np.count_nonzero(in_pml & (cell_mat != 0))),
    )
    if nm and max(max(m["eps_order"], m["mu_order"]) for m in mats) > MAX_ORDER:
        raise UnsupportedFeature("Z-filter order above %d" % MAX_ORDER)

    # excitation functions + point excitations
    val, valf = excitation_tables(spec.functions, nsteps, dt)
    pts = centre_pts
    tables.update(
        n_functions=len(spec.functions), fn_value=val, fn_value_face=valf,
        n_exc_points=len(pts),
        pt_cell=np.array([exc_number[(p.cell[2] - 1) * nx * ny + (p.cell[1] - 1) * nx + p.cell[0] - 1] for p in pts],
                         dtype=np.int32),
        pt_comp=np.array([COMPONENTS[p.component] for p in pts], dtype=np.int32),
        pt_fn=np.array([p.function for p in pts], dtype=np.int32),
        pt_type=np.array([p.source_type for p in pts], dtype=np.int32),
        n_exc_cells=int(cell_exc.sum()),
    )

    # special faces: Huygens and face-point excitation faces, DFT and
    # face-point output faces, in connect order
    face_exc = {}
    face_out = {}

    def face_key(q):
        (ox, oy, oz), axis, side = FACE_POINT[q.face]
        return ((q.cell[0] + ox, q.cell[1] + oy, q.cell[2] + oz), axis), side

    face_pts = [(q, *face_key(q)) for q in spec.point_excitations if q.face != "centre"]
    face_probes = [(q, *face_key(q)) for q in spec.outputs if q.face != "centre"]
    for _, key, _ in face_pts:
        face_exc[key] = True
    for _, key, _ in face_probes:
        face_out[key] = True
    hs = spec.huygens
    outer = isinstance(hs, HuygensOuter)
    hs_patches = _huygens_patches(hs) if hs is not None and not outer else []
    if hs is not None and not outer and not hs_patches:
        raise ValueError("empty Huygens patch: r0 and r1 are (min, max) cell ranges")

    def connect_key(c, code):  # a cell face -> (cell whose min face it is, axis)
        axis = (code - 1) % 3
        if code <= 3:
            return (tuple(c), axis + 1)
        c = list(c)
        c[axis] += 1
        return (tuple(c), axis + 1)

    for c, code in hs_patches:
        face_exc[connect_key(c, code)] = True
    ff_faces = [ff.faces() for ff in spec.far_field_surfaces]
    for fl in ff_faces:
        for c, code in fl:
            face_out[connect_key(c, code)] = True
    os_faces = [os_.faces() for os_ in spec.output_surfaces]
    for fl in os_faces:
        for c, code in fl:
            face_out[connect_key(c, code)] = True
    ps_faces = [ps.faces() for ps in spec.power_surfaces]
    mode_faces = [mo.faces() for mo in spec.mode_outputs]
    for fl in ps_faces + mode_faces:
        for c, code in fl:
            face_out[connect_key(c, code)] = True
    rcs_faces = spec.rcs_surface.faces() if spec.rcs_surface is not None else []
    for c, code in rcs_faces:
        face_out[connect_key(c, code)] = True
    dft_faces = [ds.faces() for ds in spec.dft_surfaces]
    for fl in dft_faces:
        for c, code in fl:
            face_out[connect_key(c, code)] = True
    face_mat, face_smat = {}, {}
    for sh in spec.surface_sheets:
        if sh.kind not in SURFACE_SHEET_TYPES:
            raise UnsupportedFeature(f"surface material {sh.kind!r}: only PEC, PMC, free-space and dispersive "
                                     "sheets")
        if sh.kind == "dispersive" and not 1 <= sh.material <= len(spec.thin_layers):
            raise ValueError(f"dispersive sheet: thin-layer material {sh.material} is not defined")
        for key, sg in zip(sh.face_keys(), sh.face_signs()):  # the last sheet on a face wins
            face_mat[key] = SURFACE_SHEET_TYPES[sh.kind]
            face_smat[key] = sg * sh.material if sh.kind == "dispersive" else 0
    # connect visits the internal faces only (connect.F90:180-213: cx, cy,
    # cz .ne. 1), so a surface material on a face of the outer boundary
    # changes nothing: such faces are dropped
    for key in [k for k in face_mat if not 1 < k[0][k[1] - 1] <= (nx, ny, nz)[k[1] - 1]]:
        del face_mat[key]
        face_smat.pop(key, None)
    keys = set(face_exc) | set(face_out) | set(face_mat)
    for (c, axis) in keys:
        if c[axis - 1] <= 1 or c[axis - 1] > (nx, ny, nz)[axis - 1]:
            raise UnsupportedFeature("special face on the outer boundary")
    # connect order: cz, cy, cx, then x-, y-, z-face
    ordered = sorted(keys, key=lambda k: (k[0][2], k[0][1], k[0][0], k[1]))
    fexc_num, fout_num = {}, {}
    ne = no = 0
    face_cx, face_cy, face_cz, face_dir, face_e, face_o = [], [], [], [], [], []
    for key in ordered:
        (cx, cy, cz), axis = key
        e = o = 0
        if key in face_exc:
            ne += 1
            e = ne
            fexc_num[key] = ne
        if key in face_out:
            no += 1
            o = no
            fout_num[key] = no
        face_cx.append(cx); face_cy.append(cy); face_cz.append(cz); face_dir.append(axis)
        face_e.append(e); face_o.append(o)
    tables.update(
        n_face_points=len(face_pts),
        fpt_face=np.array([fexc_num[k] for _, k, _ in face_pts], dtype=np.int32),
        fpt_comp=np.array([COMPONENTS[q.component] for q, _, _ in face_pts], dtype=np.int32),
        fpt_fn=np.array([q.function for q, _, _ in face_pts], dtype=np.int32),
        fpt_type=np.array([q.source_type for q, _, _ in face_pts], dtype=np.int32),
        fpt_side=np.array([side if q.one_side else 0 for q, _, side in face_pts], dtype=np.int32),
        fpt_scale=np.array([q.scale for q, _, _ in face_pts], dtype=np.float64),
        n_face_probes=len(face_probes),
        fprobe_face=np.array([fout_num[k] for _, k, _ in face_probes], dtype=np.int32),
        fprobe_side=np.array([sd for _, _, sd in face_probes], dtype=np.int32),
        fprobe_comp=np.array([COMPONENTS[q.component] for q, _, _ in face_probes], dtype=np.int32))
    for q, _, _ in face_probes:
        if COMPONENTS[q.component] > 6:
            raise ValueError("a face output point records E or H (components 1..6)")
    tables["face_mat"] = np.array([face_mat.get(k, 0) for k in ordered], dtype=np.int32)
    tables["wrap"] = np.array([int(bool(v)) for v in spec.wrap], dtype=np.int32)
    if any(spec.wrap) and isinstance(spec.huygens, HuygensOuter):
        raise UnsupportedFeature("an outer-boundary Huygens surface with wrapping boundaries")
    # thin layers: the signed material per special face (positive: reversed)
    # and the filters of every thin-layer material
    tables["face_smat"] = np.array([face_smat.get(k, 0) for k in ordered], dtype=np.int32)
    MOs = MAX_ORDER + 1
    smc = [surface_material_coefficients(sm, dt) for sm in spec.thin_layers]
    tables.update(n_smat=len(smc),
                  smat_f=np.array([c["f"] for c in smc], dtype=np.float64).reshape(-1, 3, 4),
                  smat_a=np.array([c["a"] for c in smc], dtype=np.float64).reshape(-1, 3, 4, MOs),
                  smat_b=np.array([c["b"] for c in smc], dtype=np.float64).reshape(-1, 3, 4, MOs),
                  smat_order=np.array([c["order"] for c in smc], dtype=np.int32).reshape(-1, 3, 4))
    tables.update(n_faces=len(ordered), face_cx=np.array(face_cx, dtype=np.int32),
                  face_cy=np.array(face_cy, dtype=np.int32), face_cz=np.array(face_cz, dtype=np.int32),
                  face_dir=np.array(face_dir, dtype=np.int32), face_exc=np.array(face_e, dtype=np.int32),
                  face_out=np.array(face_o, dtype=np.int32), n_exc_faces=ne, n_out_faces=no)

    # Huygens surface data, huygens_surface.F90:247-715
    if outer:
        K, Ei, Hi = huygens_vectors(hs.ktheta, hs.kphi, hs.etheta, hs.ephi, hs.wave_impedance)
        cells = []  # huygens_surface.F90:517-612 order
        for cz in range(1, nz + 1):
            for cy in range(1, ny + 1):
                cells += [(1, cy, cz, FACE_XMIN), (nx, cy, cz, FACE_XMAX)]
        for cz in range(1, nz + 1):
            for cx in range(1, nx + 1):
                cells += [(cx, 1, cz, FACE_YMIN), (cx, ny, cz, FACE_YMAX)]
        cells += [(cx, cy, 1, FACE_ZMIN) for cy in range(1, ny + 1) for cx in range(1, nx + 1)]
        cells += [(cx, cy, nz, FACE_ZMAX) for cy in range(1, ny + 1) for cx in range(1, nx + 1)]
        xmin0, ymin0, zmin0 = spec.origin
        norms, offsets = [], []
        for (cx, cy, cz, code) in cells:
            axis = (code - 1) % 3
            n = [0, 0, 0]
            n[axis] = -1 if code <= 3 else 1
            off = [-0.5, -0.5, -0.5]
            off[axis] = -1.0 if code <= 3 else 0.0
            x = xmin0 + (cx + off[0]) * dl
            y = ymin0 + (cy + off[1]) * dl
            z = zmin0 + (cz + off[2]) * dl
            norms.extend(n)
            offsets.append(K[0] * x + K[1] * y + K[2] * z)
        # the extents are the mesh's own (huygens_surface.F90:508-515)
        bx, by, bz = (xmin0, xmin0 + nx * dl), (ymin0, ymin0 + ny * dl), (zmin0, zmin0 + nz * dl)
        offset_min = 1e30
        for (xx_, yy_, zz_) in ((bx[0], by[0], bz[0]), (bx[1], by[0], bz[0]), (bx[0], by[1], bz[0]),
                                (bx[1], by[1], bz[0]), (bx[0], by[0], bz[1]), (bx[1], by[0], bz[1]),
                                (bx[0], by[1], bz[1]), (bx[1], by[1], bz[1])):
            offset_min = min(K[0] * xx_ + K[1] * yy_ + K[2] * zz_, offset_min)
        tables.update(hs_n=len(cells), hs_face_exc=np.zeros(len(cells), np.int32),
                      hs_norm=np.array(norms, dtype=np.int32), hs_offset=np.array(offsets),
                      hs_Ei=np.array(Ei), hs_Hi=np.array(Hi), hs_offset_min=offset_min - dl / 2.0,
                      hs_c=C0 / spec.reduced_c, hs_fn=hs.function, hs_outer=1,
                      hs_cell=np.array(cells, dtype=np.int32).reshape(-1))
    elif hs is not None:
        K, Ei, Hi = huygens_vectors(hs.ktheta, hs.kphi, hs.etheta, hs.ephi, hs.wave_impedance)
        norms, offsets, fexc = [], [], []
        xmin0, ymin0, zmin0 = spec.origin
        cents = []
        for (c, code) in hs_patches:
            axis = (code - 1) % 3
            n = [0, 0, 0]
            n[axis] = -1 if code <= 3 else 1
            # get_cell_point_coordinate, general_mesh_subroutines.F90:84-140
            off = [-0.5, -0.5, -0.5]
            off[axis] = -1.0 if code <= 3 else 0.0
            x = xmin0 + (c[0] + off[0]) * dl
            y = ymin0 + (c[1] + off[1]) * dl
            z = zmin0 + (c[2] + off[2]) * dl
            cents.append((x, y, z))
            norms.extend(n)
            offsets.append(K[0] * x + K[1] * y + K[2] * z)
            fexc.append(fexc_num[connect_key(c, code)])
        # surface mesh extents are the face-centre extents of the recorded
        # faces (build_surface_mesh.F90:120-160); both sides of a face share
        # one centre
        cm = np.array(cents)
        bx = (cm[:, 0].min(), cm[:, 0].max())
        by = (cm[:, 1].min(), cm[:, 1].max())
        bz = (cm[:, 2].min(), cm[:, 2].max())
        offset_min = 1e30
        for (xx_, yy_, zz_) in ((bx[0], by[0], bz[0]), (bx[1], by[0], bz[0]), (bx[0], by[1], bz[0]),
                                (bx[1], by[1], bz[0]), (bx[0], by[0], bz[1]), (bx[1], by[0], bz[1]),
                                (bx[0], by[1], bz[1]), (bx[1], by[1], bz[1])):
            offset_min = min(K[0] * xx_ + K[1] * yy_ + K[2] * zz_, offset_min)
        tables.update(hs_n=len(hs_patches), hs_face_exc=np.array(fexc, dtype=np.int32),
                      hs_norm=np.array(norms, dtype=np.int32), hs_offset=np.array(offsets),
                      hs_Ei=np.array(Ei), hs_Hi=np.array(Hi), hs_offset_min=offset_min - dl / 2.0,
                      hs_c=C0 / spec.reduced_c, hs_fn=hs.function)
    else:
        tables.update(hs_n=0, hs_face_exc=np.zeros(0, np.int32), hs_norm=np.zeros(0, np.int32),
                      hs_offset=np.zeros(0), hs_Ei=np.zeros(3), hs_Hi=np.zeros(3), hs_offset_min=0.0,
                      hs_c=C0 / spec.reduced_c, hs_fn=0)

    # outputs
    tables["n_out_cells"] = int(cell_out.sum())
    tables["out_cell"] = np.array(
        [out_number[(o.cell[2] - 1) * nx * ny + (o.cell[1] - 1) * nx + o.cell[0] - 1] for o in centre_outs],
        dtype=np.int32)
    tables["out_comp"] = np.array([COMPONENTS[o.component] for o in centre_outs], dtype=np.int32)
    # geometry of the solve for host-side policies (not uploaded): 1-based
    # cells of the centre output points and point sources, PML depth per face
    tables["out_xyz"] = np.array([o.cell for o in centre_outs], dtype=np.int32).reshape(-1, 3)
    tables["pt_xyz"] = np.array([q.cell for q in centre_pts], dtype=np.int32).reshape(-1, 3)
    tables["pml_depth"] = np.array(spec.pml_cells, dtype=np.int32)
    tables["out_keep"] = point_out.reshape(-1)[cell_out.reshape(-1)].astype(np.int32)
    # 1-based output point numbers (output_points(:) order) of the centre and face points, for .tout files
    tables["out_point_no"] = np.array([i + 1 for i, q in enumerate(spec.outputs) if q.face == "centre"], dtype=np.int32)
    tables["fprobe_point_no"] = np.array([i + 1 for i, q in enumerate(spec.outputs) if q.face != "centre"],
                                         dtype=np.int32)
    # frequency output volumes: one reference volume entry per frequency
    vf, vc, v0, v1, vi, vptr, vout = [], [], [], [], [], [0], []
    for fv, vm in zip(spec.frequency_output_volumes, vol_masks):
        cells = out_number[vm.reshape(-1)]  # traversal order
        for fr in fv.frequencies:
            vf.append(fr)
            vc.append(COMPONENTS[fv.component])
            v0.append(fv.first_step)
            v1.append(nsteps if fv.last_step is None else fv.last_step)
            vi.append(fv.interval)
            vout.extend(int(c) for c in cells)
            vptr.append(len(vout))
    sf, sptr, sout = [], [0], []
    for sv, vm in zip(spec.sar_volumes, sar_masks):
        cells = out_number[vm.reshape(-1)]
        for fr in sv.frequencies:
            sf.append(fr)
            sout.extend(int(c) for c in cells)
            sptr.append(len(sout))
    tables.update(n_sar=len(sf), sar_freq=np.array(sf, dtype=np.float64), sar_cell_ptr=np.array(sptr, dtype=np.int32),
                  sar_cell_out=np.array(sout, dtype=np.int32))
    ok, oc, o0, o1, oi, optr, oout = [], [], [], [], [], [0], []
    for ov, vm in zip(spec.output_volumes, ovol_masks):
        ok.append(OUTPUT_VOLUME_KINDS[ov.kind])
        oc.append(COMPONENTS[ov.component])
        o0.append(ov.first_step)
        o1.append(nsteps if ov.last_step is None else ov.last_step)
        oi.append(ov.interval)
        oout.extend(int(c) for c in out_number[vm.reshape(-1)])
        optr.append(len(oout))
    tables.update(n_ovol=len(ok), ovol_kind=np.array(ok, dtype=np.int32), ovol_comp=np.array(oc, dtype=np.int32),
                  ovol_first=np.array(o0, dtype=np.int32), ovol_last=np.array(o1, dtype=np.int32),
                  ovol_interval=np.array(oi, dtype=np.int32), ovol_cell_ptr=np.array(optr, dtype=np.int32),
                  ovol_cell_out=np.array(oout, dtype=np.int32))
    tables.update(n_vdft=len(vf), vdft_freq=np.array(vf, dtype=np.float64), vdft_comp=np.array(vc, dtype=np.int32),
                  vdft_first=np.array(v0, dtype=np.int32), vdft_last=np.array(v1, dtype=np.int32),
                  vdft_interval=np.array(vi, dtype=np.int32), vdft_cell_ptr=np.array(vptr, dtype=np.int32),
                  vdft_cell_out=np.array(vout, dtype=np.int32))

    # DFT surfaces: one reference surface entry per frequency
    freqs, comps, ptr, fo, fs, gate = [], [], [0], [], [], []
    for ds, faces in zip(spec.dft_surfaces, dft_faces):
        if ds.first_step < 1 or ds.interval < 1:
            raise ValueError("frequency output surface first step and interval must be at least 1")
        for fr in ds.frequencies:
            freqs.append(fr)
            comps.append(COMPONENTS[ds.component])
            gate.append((ds.first_step, nsteps if ds.last_step is None else ds.last_step, ds.interval))
            for c, code in faces:  # the face code says which side's field the entry reads
                fo.append(fout_num[connect_key(c, code)])
                fs.append(code)
            ptr.append(len(fo))
    tables.update(n_dft=len(freqs), dft_freq=np.array(freqs, dtype=np.float64),
                  dft_comp=np.array(comps, dtype=np.int32), dft_face_ptr=np.array(ptr, dtype=np.int32),
                  dft_face_out=np.array(fo, dtype=np.int32), dft_face_side=np.array(fs, dtype=np.int32),
                  dft_first=np.array([g[0] for g in gate], dtype=np.int32),
                  dft_last=np.array([g[1] for g in gate], dtype=np.int32),
                  dft_interval=np.array([g[2] for g in gate], dtype=np.int32))
    # far-field surfaces: one reference surface entry per frequency
    ffreq, fptr, ffo, ffc = [], [0], [], []
    for ff, fl in zip(spec.far_field_surfaces, ff_faces):
        for fr in ff.frequencies:
            ffreq.append(fr)
            for c, code in fl:
                ffo.append(fout_num[connect_key(c, code)])
                ffc.append(code)
            fptr.append(len(ffo))
    # time-domain output surfaces
    oc, o0, o1, oi, ob, optr, ofo, ofc = [], [], [], [], [], [0], [], []
    for os_, fl in zip(spec.output_surfaces, os_faces):
        if os_.component not in SURFACE_COMPONENTS:
            raise ValueError(f"output surface component {os_.component!r}")
        if os_.first_step < 1 or os_.interval < 1:
            raise ValueError("output surface first step and interval must be >= 1")
        oc.append(SURFACE_COMPONENTS[os_.component])
        o0.append(os_.first_step)
        o1.append(nsteps if os_.last_step is None else os_.last_step)
        oi.append(os_.interval)
        ob.append(1 if os_.both_sides else 0)
        for c, code in fl:
            ofo.append(fout_num[connect_key(c, code)])
            ofc.append(code)
        optr.append(len(ofo))
    tables.update(n_osurf=len(oc), osurf_comp=np.array(oc, dtype=np.int32), osurf_first=np.array(o0, dtype=np.int32),
                  osurf_last=np.array(o1, dtype=np.int32), osurf_interval=np.array(oi, dtype=np.int32),
                  osurf_both=np.array(ob, dtype=np.int32), osurf_face_ptr=np.array(optr, dtype=np.int32),
                  osurf_face_out=np.array(ofo, dtype=np.int32), osurf_face_code=np.array(ofc, dtype=np.int32))
    # frequency-domain power surfaces: one entry per frequency
    pf, pptr, pfo, pfc = [], [0], [], []
    for ps, fl in zip(spec.power_surfaces, ps_faces):
        for fr in ps.frequencies:
            pf.append(fr)
            for c, code in fl:
                pfo.append(fout_num[connect_key(c, code)])
                pfc.append(code)
            pptr.append(len(pfo))
    tables.update(n_ps=len(pf), ps_freq=np.array(pf, dtype=np.float64), ps_face_ptr=np.array(pptr, dtype=np.int32),
                  ps_face_out=np.array(pfo, dtype=np.int32), ps_face_code=np.array(pfc, dtype=np.int32))
    # mode outputs
    mc, mptr, mfo, mfc, mw = [], [0], [], [], []
    for mo, fl in zip(spec.mode_outputs, mode_faces):
        if COMPONENTS.get(mo.component, 0) not in range(1, 7):
            raise ValueError("a mode output samples Ex..Hz")
        mc.append(COMPONENTS[mo.component])
        for (c, code), w in zip(fl, mo.weights()):
            mfo.append(fout_num[connect_key(c, code)])
            mfc.append(code)
            mw.append(w)
        mptr.append(len(mfo))
    tables.update(n_modes=len(mc), mode_comp=np.array(mc, dtype=np.int32), mode_face_ptr=np.array(mptr, dtype=np.int32),
                  mode_face_out=np.array(mfo, dtype=np.int32), mode_face_code=np.array(mfc, dtype=np.int32),
                  mode_field=np.array(mw, dtype=np.float64))
    # the RCS surface, initialise_rcs_surfaces (RCS_surfaces.F90:159-360)
    if spec.rcs_surface is not None:
        rs = spec.rcs_surface
        theta, phi = (math.pi / 180.0) * rs.theta, (math.pi / 180.0) * rs.phi
        K = (1.0 * math.sin(theta) * math.cos(phi), 1.0 * math.sin(theta) * math.sin(phi), 1.0 * math.cos(theta))
        xmin0, ymin0, zmin0 = spec.origin
        dist = []
        for c, code in rcs_faces:
            # get_cell_point_coordinate, general_mesh_subroutines.F90:84-140
            off = [-0.5, -0.5, -0.5]
            off[(code - 1) % 3] = -1.0 if code <= 3 else 0.0
            x = xmin0 + c[0] * dl + dl * off[0]
            y = ymin0 + c[1] * dl + dl * off[1]
            z = zmin0 + c[2] * dl + dl * off[2]
            dist.append(K[0] * x + K[1] * y + K[2] * z)
        dmin, dmax = min(dist), max(dist)
        # the problem file's simulation_time, or n_timesteps dt for a spec without one
        sim = spec.simulation_time if spec.simulation_time is not None else nsteps * dt
        period = (dmax - dmin) / C0 + sim
        distance = period * C0
        tables.update(rcs_on=1, rcs_theta=theta, rcs_phi=phi, rcs_npc=RCS_POINTS_PER_CELL,
                      rcs_points=int(RCS_POINTS_PER_CELL * distance / dl + 2),
                      rcs_offset=int(RCS_POINTS_PER_CELL * dmin / dl - 1),
                      rcs_face_out=np.array([fout_num[connect_key(c, code)] for c, code in rcs_faces], dtype=np.int32),
                      rcs_face_code=np.array([code for _, code in rcs_faces], dtype=np.int32),
                      rcs_face_dist=np.array(dist, dtype=np.float64))
    else:
        tables.update(rcs_on=0)
    tables.update(n_ff=len(ffreq), ff_freq=np.array(ffreq, dtype=np.float64),
                  ff_face_ptr=np.array(fptr, dtype=np.int32), ff_face_out=np.array(ffo, dtype=np.int32),
                  ff_face_code=np.array(ffc, dtype=np.int32))
    n_small, small = spec.small_to_zero if spec.small_to_zero else (0, 0.0)
    if n_small < 0 or small < 0.0:
        raise ValueError("set_small_to_zero needs n >= 0 and a value >= 0")
    tables.update(n_small_to_zero=int(n_small), small_to_zero_value=float(small))
    return tables


def probe_series(tables: dict, cell_out: np.ndarray) -> np.ndarray:
    """Pick the output-point time series from cell_output_field snapshots
    (output_points.F90:463-612): cell_out is [steps, n_out_cells, 6], or
    [steps, n_kept, 6] with only the output cells that keep a series."""
    idx = tables["out_cell"] - 1
    keep = tables.get("out_keep")
    if keep is not None and cell_out.shape[1] != int(tables["n_out_cells"]):
        slot = np.cumsum(np.asarray(keep)) - 1
        idx = slot[idx]
    comp = tables["out_comp"] - 1
    return cell_out[:, idx, comp].T.copy()  # [n_points, steps]
