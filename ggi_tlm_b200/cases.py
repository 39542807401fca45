"""Seeded synthetic problems for the SCN-TLM core.

* Known-answer cases restated from the reference's own regression tests
  (TEST_DATA/TEM_PML_TEST, TEM_MATERIAL_TEST, MATERIAL_STABILITY_TEST): their
  geometry is a 1x1xN TEM cell or a 20^3 box with rectangular blocks and a
  planar Huygens patch, which voxelise exactly without the reference mesher.
* The benchmark configurations (PEC box, PML box with dielectric spheres,
  Debye slabs, batches of uneven boxes, the 512^3 PML target), generated from
  a seed.  No public dataset is involved; these stand in for the reference's
  .inp/.mesh inputs with the sizes and value ranges of the workloads.
"""
from __future__ import annotations

import math
from typing import List, Optional, Tuple

import numpy as np

from .problem import (C0, MAT_DISPERSIVE, Block, DFTSurface, ExcitationFunction, HuygensBox, HuygensPlane,
                      OutputPoint,
                      PointExcitation, ProblemSpec, Sfilter, Sphere, VolumeMaterial, nint)


def _dt(dl: float) -> float:
    return dl / (2.0 * C0)


# ---------------------------------------------------------------------------
# Known-answer cases (reference regression tests)
# ---------------------------------------------------------------------------
def _tem_cell(nz: int, pml: bool, material: Optional[VolumeMaterial]) -> ProblemSpec:
    """TEM cell of TEST_DATA/TEM_PML_TEST and TEM_MATERIAL_TEST: one cell of
    0.1 m cross-section with PMC/PEC side walls, a +z Gaussian plane wave
    launched from a Huygens patch at z=0.1 m, Ey/Hx probes at z=9.95/10.05 m."""
    dl = 0.1
    n = nint(30e-8 / _dt(dl))
    spec = ProblemSpec(
        nx=1, ny=1, nz=nz, dl=dl, n_timesteps=n,
        R=(1.0, 1.0, -1.0, -1.0, 0.0, -1.0 if pml else 0.0), origin=(-0.05, -0.05, 0.0),
        pml_cells=(0, 0, 0, 0, 0, 20) if pml else (0,) * 6, pml_r=(0.1, 0.1, 0.1, 0.1, 0.1, 1e-4), pml_order=2,
        functions=[ExcitationFunction("gaussian", (1.0, 2e-9, 8e-9))],
        huygens=HuygensPlane(axis=3, index=1, r0=(1, 1), r1=(1, 1), function=1, ktheta=0.0, kphi=90.0,
                             etheta=1.0, ephi=0.0, side=1),
        outputs=[OutputPoint((1, 1, 100), "Ey"), OutputPoint((1, 1, 100), "Hx"), OutputPoint((1, 1, 101), "Ey"),
                 OutputPoint((1, 1, 101), "Hx")])
    if material is not None:
        spec.materials = [material]
        spec.material_regions = [(1, Block(1, 1, 1, 1, 201, 600))]
    return spec


def debye_2() -> VolumeMaterial:
    """TEST_DATA/MATERIAL_DATA/debye_2.vmat: eps(s)=(4+0.75 s/w)/(1+0.5 s/w), w=1e7."""
    return VolumeMaterial(MAT_DISPERSIVE, Sfilter(1e7, [4.0, 0.75], [1.0, 0.5]), 0.0, Sfilter(1e7, [1.0], [1.0]), 0.0)


def kat_tem_pml() -> ProblemSpec:
    """TEST_DATA/TEM_PML_TEST/PROBLEM_SPECIFICATION_FILES/TEM_cell.inp."""
    return _tem_cell(200, True, None)


def kat_tem_material() -> ProblemSpec:
    """TEST_DATA/TEM_MATERIAL_TEST/PROBLEM_SPECIFICATION_FILES/TEM_cell.inp."""
    return _tem_cell(600, False, debye_2())


def kat_material_stability() -> ProblemSpec:
    """TEST_DATA/MATERIAL_STABILITY_TEST/PROBLEM_SPECIFICATION_FILES/cavity.inp:
    20^3 box, Debye block 0.6^3 m, impulse plane wave from a 1 m^2 patch."""
    dl = 0.1
    n = nint(1e-6 / _dt(dl))
    return ProblemSpec(
        nx=20, ny=20, nz=20, dl=dl, n_timesteps=n, R=(1.0, 1.0, -1.0, -1.0, -1.0, -1.0), origin=(-1.0, -1.0, -1.0),
        materials=[debye_2()], material_regions=[(1, Block(8, 13, 8, 13, 8, 13))],
        functions=[ExcitationFunction("impulse", (1.0, 0.0))],
        huygens=HuygensPlane(axis=3, index=5, r0=(6, 15), r1=(6, 15), function=1, ktheta=0.0, kphi=90.0,
                             etheta=1.0, ephi=0.0, side=1),
        outputs=[OutputPoint((11, 11, 11), "Ey")])


def cubic_mesh_dl(xmin: float, xmax: float, n: int) -> float:
    """MESH/set_mesh_parameters.F90:61-66, dl=(dlx+dly+dlz)/3 on a cubic
    mesh, with the division by 3 evaluated as a multiplication by 1/3 as the
    reference's build flags (-funsafe-math-optimizations) compile it: for a
    4 m / 40-cell mesh this gives dl = 0.1 exactly where a true division
    gives 0.1 + 1 ulp, and the TEST_DATA/HUYGENS_SURFACE output point
    (0,0,0) then lands in cell 21 as in the golden series."""
    dlx = (xmax - xmin) / float(n)
    return (dlx + dlx + dlx) * (1.0 / 3.0)


def point_to_cell(p: float, xmin: float, dl: float) -> int:
    """MESH/general_mesh_subroutines.F90:345-383, int((p-xmin)/dl)+1, with the
    division evaluated as a multiplication by 1/dl, as the reference's build
    flags (-funsafe-math-optimizations, make_configuration_data:39) compile
    it.  The distinction matters for points on cell boundaries; the
    MATERIAL_TEST2 golden series pins it."""
    return int((p - xmin) * (1.0 / dl)) + 1


def kat_material_test2() -> ProblemSpec:
    """TEST_DATA/MATERIAL_TEST2/PROBLEM_SPECIFICATION_FILES/mat_test.inp: 60^3
    cells over 6 mm, a 1 mm cube of a Lorentz material (mur_lorentz.vmat: the
    same 2nd-order rational for eps_r and mu_r, complex poles), soft Ex
    Gaussian point source and an Ex probe 2.4 mm apart, R=0."""
    xmin, xmax, n = -3.0e-3, 3.0e-3, 60
    dl = cubic_mesh_dl(xmin, xmax, n)
    steps = nint(10e-10 / _dt(dl))
    f = Sfilter(1e10, [2.0, 3.1827e-1, 4.0518e-1], [1.0, 3.1827e-1, 4.0518e-1])
    lorentz = VolumeMaterial(MAT_DISPERSIVE, f, 0.0, Sfilter(f.wnorm, list(f.a), list(f.b)), 0.0)
    c = lambda p: point_to_cell(p, xmin, dl)  # noqa: E731
    return ProblemSpec(
        nx=n, ny=n, nz=n, dl=dl, n_timesteps=steps, R=(0.0,) * 6, origin=(xmin,) * 3,
        materials=[lorentz], material_regions=[(1, Block(26, 35, 26, 35, 26, 35))],
        functions=[ExcitationFunction("gaussian", (1.0, 1e-10, 3e-10))],
        point_excitations=[PointExcitation((c(1.2e-3), c(0.0), c(0.0)), "Ex", 1)],
        outputs=[OutputPoint((c(-1.2e-3), c(0.0), c(0.0)), "Ex")])


def pml_dielectric_slab(n: int = 40, pml: int = 8, steps: int = 300, eps_r: float = 4.0, sigma: float = 0.01,
                        slab_top: int = 15, pad: int = 0, dl: float = 5e-3) -> ProblemSpec:
    """A lossy dielectric substrate (cells z <= slab_top, every x and y) that
    runs into the PML on five sides, so its PML cells take the PML-material
    update (scatter_PML_material.F90); Gaussian Ez source in the free space
    above, Ez probes in the slab and above it, an Ex probe near the interface.
    ``pad`` > 0 surrounds the same geometry by ``pad`` free cells on every side
    and drops the PML (a reference domain whose boundary is too far away to be
    seen within ``steps``)."""
    N = n + 2 * pad
    c = N // 2 + 1
    return ProblemSpec(
        nx=N, ny=N, nz=N, dl=dl, n_timesteps=steps, pml_cells=(pml,) * 6 if pad == 0 else (0,) * 6,
        materials=[VolumeMaterial.dielectric(eps_r, sigma)],
        material_regions=[(1, Block(1, N, 1, N, 1, pad + slab_top))],
        functions=[ExcitationFunction("gaussian", (1.0, 0.05e-9, 0.2e-9))],
        point_excitations=[PointExcitation((c, c, pad + slab_top + 6), "Ez", 1)],
        outputs=[OutputPoint((c, c, pad + slab_top - 3), "Ez"), OutputPoint((c, c, pad + slab_top + 9), "Ez"),
                 OutputPoint((c + 4, c, pad + slab_top + 2), "Ex")])


def kat_huygens_box(component: str = "Ex") -> ProblemSpec:
    """TEST_DATA/HUYGENS_SURFACE/PROBLEM_SPECIFICATION_FILES/huygens_test.inp:
    40^3 cells over 4 m, R=0, a closed Huygens surface on the 2 m cube at the
    centre (cells 11..30 on each axis, side 1) launching a Gaussian plane
    wave along the cube diagonal (theta 54.73, phi 45 degrees, polarisation
    (1.0, 0.5)); the fields at the centre point (0,0,0) -> cell (21,21,21).
    The reference's volume and output surfaces of that input are
    post-processing only and are left out."""
    xmin, n = -2.0, 40
    dl = cubic_mesh_dl(xmin, 2.0, n)
    steps = nint(2e-8 / _dt(dl))
    c = point_to_cell(0.0, xmin, dl)
    return ProblemSpec(
        nx=n, ny=n, nz=n, dl=dl, n_timesteps=steps, R=(0.0,) * 6, origin=(xmin,) * 3,
        functions=[ExcitationFunction("gaussian", (1.0, 2e-9, 6e-9))],
        huygens=HuygensBox((11, 30), (11, 30), (11, 30), 1, 54.73, 45.0, 1.0, 0.5),
        outputs=[OutputPoint((c, c, c), component)])


KAT_CASES = {
    "tem_pml_Ey": kat_tem_pml,
    "tem_material_Ey": kat_tem_material,
    "material_stability_Ey": kat_material_stability,
    "material_test2_Ex": kat_material_test2,
    **{f"huygens_box_{f}": (lambda f=f: kat_huygens_box(f)) for f in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")},
}


# ---------------------------------------------------------------------------
# Benchmark configurations
# ---------------------------------------------------------------------------
def pec_box(n: int = 40, steps: int = 2000, seed: int = 1, dl: float = 0.01) -> ProblemSpec:
    """PEC-walled free-space box, Gaussian (0.2 ns, 1 ns) soft Ex point source
    at the centre cell, Ex/Ey/Ez probes at 4 seeded cells."""
    rng = np.random.default_rng(seed)
    src = (n // 2, n // 2, n // 2)
    probes: List[Tuple[int, int, int]] = []
    while len(probes) < 4:
        c = tuple(int(v) for v in rng.integers(1, n + 1, size=3))
        if c != src and c not in probes:
            probes.append(c)
    outs = [OutputPoint(c, comp) for c in probes for comp in ("Ex", "Ey", "Ez")]
    return ProblemSpec(nx=n, ny=n, nz=n, dl=dl, n_timesteps=steps, R=(-1.0,) * 6,
                       functions=[ExcitationFunction("gaussian", (1.0, 0.2e-9, 1e-9))],
                       point_excitations=[PointExcitation(src, "Ex", 1)], outputs=outs)


def _spheres(rng, n_spheres, dims, pml, rmin, rmax, eps_range=(2.0, 8.0), sigma_range=(0.0, 0.05)):
    mats, regions = [], []
    for i in range(n_spheres):
        r = float(rng.uniform(rmin, rmax))
        lo = [pml + r + 1 for _ in range(3)]
        hi = [d - pml - r - 1 for d in dims]
        if any(h <= l for l, h in zip(lo, hi)):
            continue
        c = [float(rng.uniform(l, h)) for l, h in zip(lo, hi)]
        eps = float(rng.uniform(*eps_range))
        sig = float(rng.uniform(*sigma_range))
        mats.append(VolumeMaterial.dielectric(eps, sig))
        regions.append((len(mats), Sphere(c[0], c[1], c[2], r)))
    return mats, regions


def pml_spheres(n: int = 256, pml: int = 8, n_spheres: int = 32, steps: int = 4000, seed: int = 2,
                dl: float = 5e-3, n_probes: int = 16, n_freq: int = 64, dft_size: int = 64,
                rmin: float = 5.0, rmax: float = 20.0) -> ProblemSpec:
    """PML-bounded box with seeded dielectric spheres (eps_r U[2,8], sigma
    U[0,0.05] S/m, kept out of the PML), a +z Gaussian plane wave from a
    Huygens patch just inside the z-min PML, probes, and an FP64 DFT surface
    of dft_size^2 faces at n_freq frequencies."""
    rng = np.random.default_rng(seed)
    mats, regions = _spheres(rng, n_spheres, (n, n, n), pml, rmin, rmax)
    lo, hi = pml + 1, n - pml
    probes = []
    while len(probes) < n_probes:
        c = tuple(int(v) for v in rng.integers(lo + 2, hi - 1, size=3))
        if c not in probes:
            probes.append(c)
    c0 = n // 2 - dft_size // 2 + 1
    dft_z = min(n - pml - 2, (3 * n) // 4)
    fmax = 0.3 * C0 / (10 * dl) * 10 / 3  # up to c/(10 dl): 10 cells per wavelength
    freqs = list(np.linspace(0.05 * fmax, fmax, n_freq)) if n_freq else []
    spec = ProblemSpec(
        nx=n, ny=n, nz=n, dl=dl, n_timesteps=steps, R=(0.0,) * 6, pml_cells=(pml,) * 6, pml_r=(1e-4,) * 6,
        pml_order=2, materials=mats, material_regions=regions,
        functions=[ExcitationFunction("gaussian", (1.0, 0.2e-9, 1e-9))],
        huygens=HuygensPlane(axis=3, index=pml + 1, r0=(lo, hi), r1=(lo, hi), function=1, ktheta=0.0, kphi=90.0,
                             etheta=1.0, ephi=0.0, side=1),
        outputs=[OutputPoint(c, "Ey") for c in probes],
        dft_surfaces=[DFTSurface(axis=3, index=dft_z, r0=(c0, c0 + dft_size - 1), r1=(c0, c0 + dft_size - 1),
                                 frequencies=freqs, component="Ey")] if n_freq else [])
    return spec


def debye_slabs(nx: int = 384, ny: int = 384, nz: int = 192, pml: int = 10, n_slabs: int = 6, thickness: int = 8,
                steps: int = 6000, seed: int = 3, dl: float = 2e-3, n_freq: int = 64, dft_size: int = 64,
                margin: int = 10) -> ProblemSpec:
    """PML box with z-normal 2-pole Debye slabs (eps_inf U[2,5], delta_eps
    U[5,40], tau log-U[1e-11,1e-9] s) kept out of the PML, a +z Gaussian plane
    wave, Ey probes in front of and behind each slab, FP64 DFT surface."""
    rng = np.random.default_rng(seed)
    ilo, ihi = pml + 1, nx - pml
    jlo, jhi = pml + 1, ny - pml
    zlo, zhi = pml + 1, nz - pml
    hz = zlo + 3
    avail = zhi - 3 - (hz + 4)
    pitch = max(thickness + 6, avail // max(n_slabs, 1))
    mats, regions, outs = [], [], []
    ci, cj = nx // 2, ny // 2
    for s in range(n_slabs):
        z0 = hz + 4 + s * pitch
        z1 = z0 + thickness - 1
        if z1 + 3 > zhi:
            break
        eps_inf = float(rng.uniform(2.0, 5.0))
        de = [float(rng.uniform(5.0, 40.0)) for _ in range(2)]
        tau = [float(10 ** rng.uniform(-11.0, -9.0)) for _ in range(2)]
        mats.append(VolumeMaterial.debye(eps_inf, de, tau, wnorm=1e9))
        regions.append((len(mats), Block(ilo + margin, ihi - margin, jlo + margin, jhi - margin, z0, z1)))
        outs.append(OutputPoint((ci, cj, z0 - 2), "Ey"))
        outs.append(OutputPoint((ci, cj, z1 + 2), "Ey"))
    c0 = nx // 2 - dft_size // 2 + 1
    d0 = ny // 2 - dft_size // 2 + 1
    fmax = C0 / (10 * dl)
    freqs = list(np.linspace(0.05 * fmax, fmax, n_freq)) if n_freq else []
    return ProblemSpec(
        nx=nx, ny=ny, nz=nz, dl=dl, n_timesteps=steps, R=(0.0,) * 6, pml_cells=(pml,) * 6, pml_r=(1e-4,) * 6,
        pml_order=2, materials=mats, material_regions=regions,
        functions=[ExcitationFunction("gaussian", (1.0, 0.1e-9, 0.5e-9))],
        huygens=HuygensPlane(axis=3, index=hz, r0=(ilo, ihi), r1=(jlo, jhi), function=1, ktheta=0.0, kphi=90.0,
                             etheta=1.0, ephi=0.0, side=1),
        outputs=outs,
        dft_surfaces=[DFTSurface(axis=3, index=zhi - 2, r0=(c0, c0 + dft_size - 1), r1=(d0, d0 + dft_size - 1),
                                 frequencies=freqs, component="Ey")] if n_freq else [])


def pml_point_source(nx: int = 512, ny: Optional[int] = None, nz: Optional[int] = None, pml: int = 8,
                     steps: int = 1000, dl: float = 5e-3, n_spheres: int = 0, seed: int = 4,
                     n_probes: int = 4) -> ProblemSpec:
    """PML-bounded free-space box (optionally with dielectric spheres), a
    Gaussian soft Ex point source at a seeded interior cell and Ex probes:
    the 512^3 roofline target and the boxes of the batched workload."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    rng = np.random.default_rng(seed)
    dims = (nx, ny, nz)
    rmax = max(2.0, min(d - 2 * pml for d in dims) / 4.0)
    mats, regions = _spheres(rng, n_spheres, dims, pml, min(2.0, rmax), rmax)
    inside_sphere = lambda c: any(  # noqa: E731
        (c[0] - 0.5 - r.cx) ** 2 + (c[1] - 0.5 - r.cy) ** 2 + (c[2] - 0.5 - r.cz) ** 2 <= r.r ** 2 for _, r in regions)
    lo = [pml + 1 for _ in dims]
    hi = [d - pml for d in dims]

    def pick():
        for _ in range(1000):
            c = tuple(int(rng.integers(l, h + 1)) for l, h in zip(lo, hi))
            if not inside_sphere(c):
                return c
        return tuple((l + h) // 2 for l, h in zip(lo, hi))

    src = ((nx + 1) // 2, (ny + 1) // 2, (nz + 1) // 2) if not n_spheres else pick()
    if inside_sphere(src):
        src = pick()
    probes = []
    for _ in range(n_probes):
        c = pick()
        if c != src and c not in probes:
            probes.append(c)
    return ProblemSpec(
        nx=nx, ny=ny, nz=nz, dl=dl, n_timesteps=steps, R=(0.0,) * 6, pml_cells=(pml,) * 6, pml_r=(1e-4,) * 6,
        pml_order=2, materials=mats, material_regions=regions,
        functions=[ExcitationFunction("gaussian", (1.0, 0.2e-9, 1e-9))],
        point_excitations=[PointExcitation(src, "Ex", 1)], outputs=[OutputPoint(c, "Ex") for c in probes])


def batch_boxes(n_boxes: int = 96, edge: Tuple[int, int] = (24, 160), steps: Tuple[int, int] = (1500, 5000),
                pml: int = 8, max_spheres: int = 8, seed: int = 5, dl: float = 5e-3) -> List[ProblemSpec]:
    """The batched workload: uneven PML boxes, edges U[24,160] per axis, 0-8
    dielectric spheres, a seeded Gaussian point source, steps U[1500,5000]."""
    rng = np.random.default_rng(seed)
    out = []
    for b in range(n_boxes):
        nx, ny, nz = (int(v) for v in rng.integers(edge[0], edge[1] + 1, size=3))
        st = int(rng.integers(steps[0], steps[1] + 1))
        ns = int(rng.integers(0, max_spheres + 1))
        out.append(pml_point_source(nx, ny, nz, pml=pml, steps=st, dl=dl, n_spheres=ns,
                                    seed=int(rng.integers(0, 2 ** 31)), n_probes=2))
    return out


def serving_requests(n_requests: int = 64, edge: Tuple[int, int] = (32, 256), steps: Tuple[int, int] = (1000, 8000),
                     pml: Tuple[int, int] = (6, 10), max_slabs: int = 3, seed: int = 6,
                     dl: float = 2e-3) -> List[ProblemSpec]:
    """The serving workload: mesh edges log-uniform in [32,256] per axis,
    0-3 z-normal 2-pole Debye slabs, 6-10 cell PML, 1000-8000 steps, a
    Gaussian point source and probes, FP64 DFT on a small surface."""
    rng = np.random.default_rng(seed)
    out = []
    lo, hi = math.log(edge[0]), math.log(edge[1])
    for r in range(n_requests):
        nx, ny, nz = (int(round(math.exp(rng.uniform(lo, hi)))) for _ in range(3))
        st = int(rng.integers(steps[0], steps[1] + 1))
        p = int(rng.integers(pml[0], pml[1] + 1))
        ns = int(rng.integers(0, max_slabs + 1))
        spec = pml_point_source(nx, ny, nz, pml=p, steps=st, dl=dl, n_spheres=0, seed=int(rng.integers(0, 2 ** 31)),
                                n_probes=2)
        # Debye slabs across the interior, kept out of the PML and away from the source
        zlo, zhi = p + 2, nz - p - 1
        src_z = spec.point_excitations[0].cell[2]
        for s in range(ns):
            z0 = int(rng.integers(zlo, max(zlo + 1, zhi - 2)))
            z1 = min(z0 + 2, zhi)
            if z0 <= src_z <= z1 or z1 < z0:
                continue
            eps_inf = float(rng.uniform(2.0, 5.0))
            de = [float(rng.uniform(5.0, 40.0)) for _ in range(2)]
            tau = [float(10 ** rng.uniform(-11.0, -9.0)) for _ in range(2)]
            spec.materials.append(VolumeMaterial.debye(eps_inf, de, tau, wnorm=1e9))
            spec.material_regions.append((len(spec.materials), Block(p + 1, nx - p, p + 1, ny - p, z0, z1)))
        # drop probes that fell inside a slab (the reference warns but allows it; keep them in free space)
        out.append(spec)
    return out
