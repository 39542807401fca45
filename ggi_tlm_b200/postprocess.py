"""Result files computed on the host from the device accumulators.

The time loop leaves frequency-domain accumulators on the device (far-field
J and M per face, SAR field DFTs per cell); after the run the reference
turns them into its result files.  These are the same computations, in the
reference's formulas and file formats, on the arrays the library returns:

- far-field patterns, ``write_far_field_surfaces``
  (OUTPUT/far_field_surfaces.F90:370-712): per far-field surface and
  (theta, phi), the radiation integrals N, L over the surface faces
  (Balanis' 3D form; the 2D form about z) and |E_theta|, |E_phi| at 1 m, in
  ``NAME.far_field.fout.<surface>``;
- SAR, ``write_SAR_volumes`` (OUTPUT/SAR_volumes.F90:334-622): per SAR
  volume the sum over its cells of |E|^2 / 2 times the conductivity and the
  cell volume, divided by the volume's mass, in ``NAME.SAR.fout``;
- the RCS, ``write_rcs_surfaces`` (OUTPUT/RCS_surfaces.F90:575-762): the
  monostatic far field in time (``NAME.rcs.tout``) and its spectrum
  against the incident field's (``NAME.rcs.fout``).
"""
from __future__ import annotations

import math
import os
from typing import List, Optional, Sequence, Tuple

import numpy as np

from .problem import C0, PI, Z0
from .tout import fortran_e


def face_point(origin: Sequence[float], dl: float, cell: Sequence[int], code: int) -> Tuple[float, float, float]:
    """get_cell_point_coordinate (MESH/general_mesh_subroutines.F90:84-135):
    the centre of face ``code`` (1..6: xmin, ymin, zmin, xmax, ymax, zmax) of
    the 1-based ``cell``, or the cell centre for code 7."""
    off = [-0.5, -0.5, -0.5]
    if 1 <= code <= 6:
        off[(code - 1) % 3] = -1.0 if code <= 3 else 0.0
    return tuple(origin[a] + cell[a] * dl + dl * off[a] for a in range(3))


def _angles(lo: float, hi: float, step: float) -> np.ndarray:
    """The reference's angle loop after read_far_field_surface converts the
    degrees to radians: int((max - min) / step) + 1 values min + (n - 1) step."""
    a0, a1, da = (PI / 180.0) * lo, (PI / 180.0) * hi, (PI / 180.0) * step
    n = int((a1 - a0) / da) + 1
    return np.array([a0 + k * da for k in range(n)])


def far_field_pattern(acc: np.ndarray, points: np.ndarray, frequency: float, dl: float, theta, phi,
                      dim: int = 3):
    """|E_theta| and |E_phi| at r0 = 1 m from one far-field surface's
    accumulators ``acc`` [faces, 6] (complex J_x, J_y, J_z, M_x, M_y, M_z)
    and face centres ``points`` [faces, 3]; ``theta`` and ``phi`` are
    (min, max, step) in degrees.  Returns (theta, phi) in radians [n] and
    |E_theta|, |E_phi| [n], theta outer and phi inner as the reference
    loops."""
    beta = 2.0 * PI * frequency / C0
    jbeta = 1j * beta
    r0 = 1.0
    J, M = acc[:, 0:3], acc[:, 3:6]
    if dim == 2:
        dA = dl
        prop2 = np.sqrt(jbeta / (8.0 * PI * r0)) * np.exp(jbeta * r0)
        th = np.array([PI / 2.0])
    else:
        dA = dl * dl
        prop2 = jbeta * np.exp(jbeta * r0) / (4.0 * PI * r0)
        th = _angles(*theta)
    ph = _angles(*phi)
    out_t, out_p, et, ep = [], [], [], []
    for t in th:
        ct, st = math.cos(t), math.sin(t)
        for p in ph:
            cp, sp = math.cos(p), math.sin(p)
            r = np.array([r0 * st * cp, r0 * st * sp, r0 * ct])  # rthetaphi_to_xyz_point
            if dim == 2:
                rp_cos = points[:, 0] * r[0] + points[:, 1] * r[1]
            else:
                rp_cos = points @ r
            prop = np.exp(jbeta * rp_cos) * dA
            if dim == 2:
                Nz = np.sum(J[:, 2] * prop)
                Nphi = np.sum((-J[:, 0] * sp + J[:, 1] * cp) * prop)
                Lz = np.sum(M[:, 2] * prop)
                Lphi = np.sum((-M[:, 0] * sp + M[:, 1] * cp) * prop)
                e_t = -prop2 * (Lphi - Z0 * Nz)  # minus the Ez component
                e_p = prop2 * (Lz + Z0 * Nphi)
            else:
                Nt = np.sum((J[:, 0] * ct * cp + J[:, 1] * ct * sp - J[:, 2] * st) * prop)
                Nphi = np.sum((-J[:, 0] * sp + J[:, 1] * cp) * prop)
                Lt = np.sum((M[:, 0] * ct * cp + M[:, 1] * ct * sp - M[:, 2] * st) * prop)
                Lphi = np.sum((-M[:, 0] * sp + M[:, 1] * cp) * prop)
                e_t = -prop2 * (Lphi + Z0 * Nt)
                e_p = prop2 * (Lt - Z0 * Nphi)
            out_t.append(t)
            out_p.append(p)
            et.append(abs(e_t))
            ep.append(abs(e_p))
    return np.array(out_t), np.array(out_p), np.array(et), np.array(ep)


def far_field_lines(theta: np.ndarray, phi: np.ndarray, et: np.ndarray, ep: np.ndarray, n_theta: int, n_phi: int,
                    dt: float, dim: int = 3) -> List[str]:
    """The far-field file: for the 3D transform a ``(A2,2I6,ES16.6)`` header
    ('# ', the theta and phi counts, 1/dt), then one ``4E14.6`` line per
    angle pair (degrees, |E_theta|, |E_phi|).  The 2D transform writes the
    lines only (the reference opens no file for it and writes to its far
    field unit as it stands; here it goes to the same numbered file)."""
    lines = []
    if dim != 2:
        lines.append("# " + f"{n_theta:6d}{n_phi:6d}" + _es(1.0 / dt, 16, 6))
    for t, p, a, b in zip(theta, phi, et, ep):
        lines.append(fortran_e(t * 180.0 / PI, 14, 6) + fortran_e(p * 180.0 / PI, 14, 6) + fortran_e(a, 14, 6) +
                     fortran_e(b, 14, 6))
    return lines


def _es(v: float, width: int, digits: int) -> str:
    """Fortran ``ESw.d``: d.ddddddE+xx, right-justified."""
    if v == 0.0:
        body = "0." + "0" * digits + "E+00"
    else:
        m, e = f"{abs(v):.{digits}e}".split("e")
        e = int(e)
        body = ("-" if v < 0 else "") + m + (f"E{'+' if e >= 0 else '-'}{abs(e):02d}" if abs(e) < 100 else
                                              f"{'+' if e >= 0 else '-'}{abs(e):03d}")
    return body.rjust(width)


def far_field_face_points(spec, t: dict) -> List[np.ndarray]:
    """Per far-field table entry (one surface and frequency), the face
    centres [faces, 3] in the order of the entry's accumulators."""
    pts = []
    for ff in spec.far_field_surfaces:
        faces = ff.faces()
        p = np.array([face_point(spec.origin, spec.dl, c, code) for c, code in faces]).reshape(-1, 3)
        for _ in ff.frequencies:
            pts.append(p)
    return pts


def write_far_field_surfaces(name: str, spec, t: dict, acc: np.ndarray, post: Sequence[dict],
                             directory: str = ".") -> List[str]:
    """Write ``<name>.far_field.fout.<k>`` for every far-field surface entry
    k (1-based, one frequency each as the .inp reader makes them); ``acc`` is
    the library's far-field accumulator array [faces of all entries, 6]
    complex and ``post`` the reader's far-field angle records."""
    written = []
    ptr = np.asarray(t["ff_face_ptr"])
    pts = far_field_face_points(spec, t)
    for k, (pinfo, p) in enumerate(zip(post, pts), start=1):
        a = acc[ptr[k - 1]:ptr[k]]
        th, ph, et, ep = far_field_pattern(a, p, pinfo["frequency"], spec.dl, pinfo["theta"], pinfo["phi"],
                                           pinfo.get("dim", 3))
        n_phi = len(_angles(*pinfo["phi"]))
        n_theta = len(th) // max(n_phi, 1)
        path = os.path.join(directory, f"{name}.far_field.fout.{k}")
        with open(path, "w") as f:
            for line in far_field_lines(th, ph, et, ep, n_theta, n_phi, float(t["dt"]), pinfo.get("dim", 3)):
                f.write(line + "\n")
        written.append(path)
    return written


def sar_values(spec, t: dict, acc: np.ndarray, densities: Sequence[float]) -> List[Tuple[float, int, float]]:
    """(frequency, SAR volume number, SAR) per SAR entry from the library's
    SAR accumulators ``acc`` [cells of all entries, 3] complex (E_x, E_y,
    E_z DFTs times dt): SAR = sigma V_cell sum_cells |E|^2 / 2 / mass with
    mass = V_cell rho n_cells (SAR_volumes.F90:195-205, 576-605).  The
    conductivity is the SAR material's sigma_e; the reference allows only
    a material with a constant permittivity and no magnetic conductivity
    (SAR_volumes.F90:150-195)."""
    ptr = np.asarray(t["sar_cell_ptr"])
    freqs = np.asarray(t["sar_freq"])
    vol = spec.dl ** 3
    rows = []
    k = 0
    for n, sv in enumerate(spec.sar_volumes, start=1):
        mat = _sar_material(spec, sv)
        for _ in sv.frequencies:
            e = acc[ptr[k]:ptr[k + 1]]
            s = 0.0
            for c in range(e.shape[0]):  # the reference's cell order, summed left to right
                s = s + 0.5 * (abs(e[c, 0]) ** 2 + abs(e[c, 1]) ** 2 + abs(e[c, 2]) ** 2)
            mass = vol * densities[n - 1] * e.shape[0]
            rows.append((float(freqs[k]), n, s * mat.sigma_e * vol / mass))
            k += 1
    return rows


def check_sar_volumes(spec) -> None:
    """Raise unless every SAR volume lies in a material of constant
    permittivity without magnetic conductivity (initialise_SAR_volumes,
    SAR_volumes.F90:150-190, stops the run otherwise)."""
    for sv in spec.sar_volumes:
        _sar_material(spec, sv)


def _sar_material(spec, sv):
    """The volume material whose cells the SAR volume covers."""
    from .problem import _region_mask

    from .problem import MAT_DISPERSIVE

    want = sv.mask(spec)
    for num, region in spec.material_regions:
        if np.array_equal(_region_mask(spec, region), want):
            m = spec.materials[num - 1]
            if m.type != MAT_DISPERSIVE:
                raise ValueError("SAR in a PEC or PMC material")
            if len(m.eps.a) != 1 or len(m.eps.b) != 1:  # filter orders above 0
                raise ValueError("SAR in a dispersive dielectric material")
            if len(m.mu.a) != 1 or len(m.mu.b) != 1:
                raise ValueError("SAR in a dispersive magnetic material")
            if m.sigma_m != 0.0:
                raise ValueError("SAR in a material with a magnetic conductivity")
            return m
    raise ValueError("a SAR volume that is not one material's cells")


def sar_line(freq: float, number: int, sar: float) -> str:
    """``write(unit,*) frequency, volume, SAR`` as gfortran's list-directed
    output writes a REAL*8, a default INTEGER (I12) and a REAL*8."""
    return (_ld_real(freq) + f"{number:12d}" + _ld_real(sar)).rstrip()


def _ld_real(v: float) -> str:
    """gfortran list-directed REAL*8, the edit descriptor 1PG26.17E3: for
    0.1 <= |v| < 1e17 F editing with 17 significant digits right-justified
    in 21 columns and 5 blanks after, else d.dddddddddddddddd with a
    three-digit exponent, right-justified in 26 columns."""
    a = abs(v)
    if v == 0.0:
        return "0.0000000000000000".rjust(21) + " " * 5
    m, e = f"{v:.16e}".split("e")
    e = int(e)
    if -1 <= e < 17:  # |v|, rounded to 17 significant digits, in [0.1, 1e17)
        k = e + 1 if a >= 1.0 else 0
        return f"{v:.{17 - k}f}".rjust(21) + " " * 5
    return (m + f"E{'+' if e >= 0 else '-'}{abs(e):03d}").rjust(26)


def write_sar_volumes(name: str, spec, t: dict, acc: np.ndarray, densities: Sequence[float],
                      directory: str = ".") -> List[str]:
    path = os.path.join(directory, name + ".SAR.fout")
    with open(path, "w") as f:
        for row in sar_values(spec, t, acc, densities):
            f.write(sar_line(*row) + "\n")
    return [path]


def rcs_lines(t: dict, far: np.ndarray, fmin: float, fmax: float, fstep: float, function: int) -> Tuple[List[str],
                                                                                                       List[str]]:
    """The RCS files of write_rcs_surfaces (RCS_surfaces.F90:575-762) from
    the library's time-domain far field ``far`` [4, n_points] (E_theta,
    E_phi, H_theta, H_phi per far-field time bin):

    - ``.rcs.tout``: per bin d its time d dl / (n_points_per_cell c0) and
      the four values, |v| < 1e-30 written as 0, format (I10,5E14.6);
    - ``.rcs.fout``: per frequency fmin + (k-1) fstep, k up to
      int((fmax-fmin)/fstep)+1, the DFT of the four series times
      j 2 pi f / c0, the incident field's DFT (the Huygens surface's
      excitation function over the run's steps) and
      RCS = 10 log10(4 pi Re(E_theta H_phi* - E_phi H_theta*) / (|Einc|^2 / Z0))
      (-1000 when not positive), format 5E14.6."""
    dl, dt = float(t["dl"]), float(t["dt"])
    npc = int(t["rcs_npc"])
    n = far.shape[1]
    tout = []
    for d in range(1, n + 1):
        tl = d * dl / (npc * C0)
        v = [0.0 if abs(x) < 1e-30 else float(x) for x in far[:, d - 1]]
        tout.append(f"{d:10d}" + fortran_e(tl, 14, 6) + "".join(fortran_e(x, 14, 6) for x in v))
    fn = np.asarray(t["fn_value"]).reshape(int(t["n_functions"]), -1)[function - 1]
    nsteps = int(t["n_timesteps"])
    dt_local = dl / (npc * C0)
    nf = int((fmax - fmin) / fstep) + 1
    fout_lines = []
    for k in range(1, nf + 1):
        f = fmin + (k - 1) * fstep
        einc = 0j
        for ts in range(1, nsteps + 1):
            einc = einc + fn[ts - 1] * (dt * np.exp(-1j * 2.0 * PI * f * ((ts - 1) * dt)))
        acc = [0j, 0j, 0j, 0j]
        for d in range(1, n + 1):
            fc = dt_local * np.exp(-1j * 2.0 * PI * f * (d * dl / (npc * C0)))
            for c in range(4):
                acc[c] = acc[c] + far[c, d - 1] * fc
        et, ep, ht, hp = (a * 1j * 2.0 * PI * f / C0 for a in acc)
        rpower = (et * np.conj(hp) - ep * np.conj(ht)).real
        ipower = abs(einc) ** 2 / Z0
        rcs = 10.0 * math.log10(4.0 * PI * rpower / ipower) if (rpower > 0.0 and ipower != 0.0) else -1000.0
        fout_lines.append("".join(fortran_e(x, 14, 6) for x in (f, abs(et), abs(ep), abs(einc), rcs)))
    return tout, fout_lines


def write_rcs(name: str, t: dict, far: np.ndarray, rcs_range: Sequence[float], function: int,
              directory: str = ".") -> List[str]:
    """Write ``<name>.rcs.tout`` and ``<name>.rcs.fout``; ``rcs_range`` is
    the packet's (fmin, fmax, fstep) and ``function`` the Huygens surface's
    excitation function number."""
    tout, fo = rcs_lines(t, far, *rcs_range, function)
    out = []
    for extn, lines in ((".rcs.tout", tout), (".rcs.fout", fo)):
        path = os.path.join(directory, name + extn)
        with open(path, "w") as f:
            for line in lines:
                f.write(line + "\n")
        out.append(path)
    return out


# The four corners of a cell face (face codes 1..6: xmin, ymin, zmin, xmax,
# ymax, zmax) as offsets from the cell's high corner in cells, in the order
# get_cell_face_corner_coordinates lists them (MESH/general_mesh_subroutines.F90:154-269).
_FACE_CORNERS = {
    1: ((-1, -1, -1), (-1, -1, 0), (-1, 0, 0), (-1, 0, -1)),
    2: ((-1, -1, -1), (0, -1, -1), (0, -1, 0), (-1, -1, 0)),
    3: ((-1, -1, -1), (-1, 0, -1), (0, 0, -1), (0, -1, -1)),
    4: ((0, -1, -1), (0, 0, -1), (0, 0, 0), (0, -1, 0)),
    5: ((-1, 0, -1), (-1, 0, 0), (0, 0, 0), (0, 0, -1)),
    6: ((-1, -1, 0), (0, -1, 0), (0, 0, 0), (-1, 0, 0)),
}
# the eight corners of a cell (get_cell_corner_coordinates, :285-330) and
# the order output_volumes.F90:416-450 writes them: six faces of four points
_CELL_CORNERS = ((-1, -1, -1), (-1, -1, 0), (-1, 0, 0), (-1, 0, -1), (0, -1, -1), (0, -1, 0), (0, 0, 0), (0, 0, -1))
_CELL_FACE_POINTS = (1, 2, 3, 4, 5, 8, 7, 6, 1, 5, 6, 2, 4, 3, 7, 8, 1, 4, 8, 5, 2, 6, 7, 3)


def _corner(origin: Sequence[float], dl: float, cell: Sequence[int], off: Sequence[int]) -> Tuple[float, ...]:
    """mesh_min + cell*dl, less dl where the offset is -1 (the reference's
    order of operations)."""
    return tuple((origin[a] + cell[a] * dl) - dl if off[a] else origin[a] + cell[a] * dl for a in range(3))


def _xyz_line(p: Sequence[float]) -> str:
    return "".join(fortran_e(v, 14, 5) for v in p)  # format(3E14.5)


def _list_int(v: int) -> str:
    return f"{int(v):12d}"  # gfortran list-directed INTEGER


def surface_field_template(number: int, spec, faces, n_frames: int) -> List[str]:
    """The template block of one output surface in ``.surface_field.tout``
    (output_surfaces.F90:532-569): point count, face count, frame count, the
    four corners of every face, then each face as four point numbers."""
    out = [f"# START SURFACE FIELD FILE TEMPLATE, OUTPUT SURFACE NUMBER:{number:5d}",
           "# Number of points:", f"{4 * len(faces):10d}", "# Number of faces:", f"{len(faces):10d}",
           "# Number of frames:", f"{n_frames:10d}"]
    for cell, code in faces:
        out += [_xyz_line(_corner(spec.origin, spec.dl, cell, off)) for off in _FACE_CORNERS[code]]
    out += [f"{4:3d}" + "".join(f"{4 * k + j:12d}" for j in range(4)) for k in range(len(faces))]
    out.append(f"# END SURFACE FIELD FILE TEMPLATE, OUTPUT SURFACE NUMBER:{number:5d}")
    return out


def frequency_output_surface_lines(spec, t: dict, dft: np.ndarray) -> List[str]:
    """``.frequency_output_surface.fout``: the entry count
    (frequency_output_surfaces.F90:265-268), then per entry (one surface and
    frequency) its template (:646-677; the four corners of every face after
    the side flip, 24 frames) and each face's cell and phasor, real,
    imaginary and magnitude (:679-696).  ``dft`` is [faces, 2] in the
    tables' entry order."""
    entries = [ds for ds in spec.dft_surfaces for _ in ds.frequencies]
    ptr = np.asarray(t["dft_face_ptr"]) if len(entries) else np.zeros(1, dtype=np.int32)
    out = ["# NUMBER OF FREQUENCY OUTPUT SURFACES:", f"{len(entries):10d}"]
    for d, ds in enumerate(entries):
        faces = ds.faces()
        if len(faces) != int(ptr[d + 1] - ptr[d]):
            raise ValueError(f"frequency output surface {d + 1}: {len(faces)} faces, tables hold {ptr[d + 1] - ptr[d]}")
        out += [f"# START SURFACE FIELD FILE TEMPLATE, OUTPUT SURFACE NUMBER:{d + 1:10d}",
                "# Number of points:", f"{4 * len(faces):10d}", "# Number of faces:", f"{len(faces):10d}",
                "# Number of frames:", f"{24:10d}"]
        for cell, code in faces:
            out += [_xyz_line(_corner(spec.origin, spec.dl, cell, off)) for off in _FACE_CORNERS[code]]
        out += [f"{4:3d}" + "".join(f"{4 * k + j:12d}" for j in range(4)) for k in range(len(faces))]
        for (cell, _), (re, im) in zip(faces, dft[ptr[d]:ptr[d + 1]]):
            out.append("".join(f"{int(c):8d}" for c in cell) +  # format(3I8,3E16.8)
                       fortran_e(re, 16, 8) + fortran_e(im, 16, 8) + fortran_e(abs(complex(re, im)), 16, 8))
    return out


def write_frequency_output_surfaces(name: str, spec, t: dict, dft: np.ndarray, directory: str = ".") -> List[str]:
    if not spec.dft_surfaces:
        return []
    path = os.path.join(directory, name + ".frequency_output_surface.fout")
    with open(path, "w") as f:
        for line in frequency_output_surface_lines(spec, t, dft):
            f.write(line + "\n")
    return [path]


def _output_steps(first: int, last: Optional[int], interval: int, n: int) -> List[int]:
    """get_output_flag (OUTPUT/output.F90:564-598) over timesteps 1..n."""
    hi = n if last is None else min(last, n)
    return [ts for ts in range(max(first, 1), hi + 1) if (ts - first) % interval == 0]


def surface_field_lines(spec, t: dict, values: Sequence[np.ndarray]) -> List[str]:
    """``NAME.surface_field.tout`` (output_surfaces.F90:326-327, 532-569,
    906-927): the number of output surfaces, each surface's template, then
    per output timestep, per surface that outputs on it, a frame of its face
    values (E14.5).  ``values`` holds the library's [frames, faces] array of
    each surface (``GpuMesh.output_surfaces``)."""
    n = int(t["n_timesteps"])
    surfs = spec.output_surfaces
    steps = [_output_steps(s.first_step, s.last_step, s.interval, n) for s in surfs]
    out = ["# NUMBER OF OUTPUT SURFACES", _list_int(len(surfs))]
    for k, s in enumerate(surfs, start=1):
        out += surface_field_template(k, spec, s.faces(), len(steps[k - 1]))
    frame = [0] * len(surfs)
    row_of = [{ts: i for i, ts in enumerate(st)} for st in steps]
    for ts in range(1, n + 1):
        for k in range(len(surfs)):
            if ts not in row_of[k]:
                continue
            frame[k] += 1
            vals = np.asarray(values[k])[row_of[k][ts]]
            out += ["# START OF SURFACE FIELD OUTPUT DATA", "# OUTPUT SURFACE NUMBER", _list_int(k + 1),
                    "# FRAME NUMBER", _list_int(frame[k]), "# NUMBER OF FACES", _list_int(len(vals)),
                    "# SURFACE FIELD DATA"]
            out += [fortran_e(v, 14, 5) for v in vals]
            out.append(f"# END OF SURFACE FIELD OUTPUT DATA, OUTPUT SURFACE NUMBER:{k + 1:5d}")
    return out


def volume_field_lines(spec, t: dict, values: Sequence[np.ndarray]) -> List[str]:
    """``NAME.volume_field.tout`` (output_volumes.F90:227-228, 403-465,
    718-745) for the output volumes of kind "field", numbered in order: each
    volume's template (24 corner points and six 4-point faces a cell, cells
    in traversal order as the mesher lists them), then per output timestep a
    frame with each cell's value written once per face.  ``values`` is
    ``GpuMesh.output_volumes()`` (all kinds, in the spec's order)."""
    n = int(t["n_timesteps"])
    vols = [(k, v) for k, v in enumerate(spec.output_volumes) if v.kind == "field"]
    out = ["# NUMBER OF OUTPUT VOLUMES", _list_int(len(vols))]
    steps, cells = [], []
    for num, (k, v) in enumerate(vols, start=1):
        st = _output_steps(v.first_step, v.last_step, v.interval, n)
        zz, yy, xx = np.nonzero(v.mask(spec))
        cl = [(int(x) + 1, int(y) + 1, int(z) + 1) for z, y, x in zip(zz, yy, xx)]
        steps.append(st)
        cells.append(cl)
        out += [f"# START volume FIELD FILE TEMPLATE, OUTPUT volume NUMBER:{num:5d}", "# Number of points:",
                f"{24 * len(cl):10d}", "# Number of faces:", f"{6 * len(cl):10d}", "# Number of frames:",
                f"{len(st):10d}"]
        for c in cl:
            out += [_xyz_line(_corner(spec.origin, spec.dl, c, _CELL_CORNERS[q - 1])) for q in _CELL_FACE_POINTS]
        out += [f"{4:3d}" + "".join(f"{4 * f + j:12d}" for j in range(4)) for f in range(6 * len(cl))]
        out.append(f"# END VOLUME FIELD FILE TEMPLATE, OUTPUT VOLUME NUMBER:{num:5d}")
    frame = [0] * len(vols)
    row_of = [{ts: i for i, ts in enumerate(st)} for st in steps]
    for ts in range(1, n + 1):
        for j, (k, _) in enumerate(vols):
            if ts not in row_of[j]:
                continue
            frame[j] += 1
            vals = np.asarray(values[k])[row_of[j][ts]]
            out += ["# START OF VOLUME FIELD OUTPUT DATA", "# OUTPUT VOLUME NUMBER", _list_int(j + 1),
                    "# FRAME NUMBER", _list_int(frame[j]), "# NUMBER OF cellS", _list_int(6 * len(vals)),
                    "# volume FIELD DATA"]
            for v in vals:
                out += [fortran_e(v, 14, 5)] * 6
            out.append(f"# END OF VOLUME FIELD OUTPUT DATA, OUTPUT volume NUMBER:{j + 1:5d}")
    return out


def write_field_files(name: str, spec, t: dict, surfaces: Optional[Sequence[np.ndarray]],
                      volumes: Optional[Sequence[np.ndarray]], directory: str = ".") -> List[str]:
    """Write ``NAME.surface_field.tout`` and ``NAME.volume_field.tout`` when
    the problem has output surfaces / field output volumes."""
    written = []
    if spec.output_surfaces and surfaces is not None:
        path = os.path.join(directory, name + ".surface_field.tout")
        with open(path, "w") as f:
            f.write("\n".join(surface_field_lines(spec, t, surfaces)) + "\n")
        written.append(path)
    if any(v.kind == "field" for v in spec.output_volumes) and volumes is not None:
        path = os.path.join(directory, name + ".volume_field.tout")
        with open(path, "w") as f:
            f.write("\n".join(volume_field_lines(spec, t, volumes)) + "\n")
        written.append(path)
    return written
