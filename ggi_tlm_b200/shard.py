"""z-slab partitioning of one mesh over several GPUs.

The reference's MPI build splits the mesh into z-slabs, one per rank
(``mesh_partition``, MESH/general_mesh_subroutines.F90:868-972: cell plane
``cz`` belongs to rank ``INT(np (cz-1) / nz)``), and exchanges two ports of
one z-plane with each neighbour twice a timestep
(TLM_SOLVER/TLM_parallel_pass_data.F90:38-279): after the scatter, the
Vx_zmax, Vy_zmax pulses of a slab's top plane go up into the ghost plane
below the next slab, whose connect then pairs them with its first plane;
after the outer boundary the connected values come back down.

Here each slab is a mesh of its own on its own GPU (``slab_tables`` cuts
the global setup tables), and the library's pull-form step needs one
exchange per timestep: before a slab's next step, the ghost plane below it
must hold the Vx_zmax, Vy_zmax pulses the slab below reflected from its top
plane, and the ghost plane above it the Vx_zmin, Vy_zmin pulses the slab
above reflected from its first plane (``tlm_gpu_halo_get`` /
``tlm_gpu_halo_put``, one z-plane of two ports each way).  ``DistShard``
drives that with ``torch.distributed`` point-to-point transfers, one rank
per slab (NCCL over NVLink between GPUs; gloo on the CPU for the tests);
``LocalShards`` holds every slab in one process.

Supported: the cell-centred path (free space, PML, volume materials, point
sources, probes, the denormal flush) and the special faces inside a slab
(Huygens surfaces, surface sheets and thin layers, face sources, face
probes, frequency output surfaces).  A special face on a z-face between two
slabs, the outer-boundary Huygens surface, whole-surface and volume outputs
(far field, output surfaces and volumes, power, modes, RCS, SAR) and z
wrapping are refused with ``UnsupportedFeature``.
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np

from .problem import UnsupportedFeature

# tables whose non-empty presence needs whole-mesh outputs or the outer boundary
_REFUSED_COUNTS = ("n_ff", "n_osurf", "n_ps", "n_modes", "rcs_on", "n_sar", "n_ovol", "n_vdft", "hs_outer")


def slab_bounds(nz: int, parts: int) -> List[Tuple[int, int]]:
    """0-based [z0, z1) of each slab: plane cz (1-based) belongs to slab
    INT(parts (cz-1) / nz), as mesh_partition assigns cell_rank."""
    if parts < 1 or parts > nz:
        raise ValueError(f"cannot split {nz} planes into {parts} slabs")
    owner = [int(parts * (cz - 1) / nz) for cz in range(1, nz + 1)]
    out = []
    for r in range(parts):
        zs = [z for z in range(nz) if owner[z] == r]
        out.append((zs[0], zs[-1] + 1))
    return out


def check_shardable(t: dict):
    for k in _REFUSED_COUNTS:
        if int(np.sum(t.get(k, 0))):
            raise UnsupportedFeature(f"z-slab sharding of a mesh with {k} > 0 (whole-surface or volume outputs, "
                                     "or the outer-boundary Huygens surface)")
    if int(np.asarray(t.get("wrap", (0, 0, 0)))[2]):
        raise UnsupportedFeature("z-slab sharding of a mesh that wraps in z")


def _range_of(flags: np.ndarray, lo: int, hi: int) -> Tuple[int, int]:
    """Numbers (0-based) that the flagged entries in [lo, hi) of a
    traversal-ordered flag array get in the global numbering."""
    before = int(np.count_nonzero(flags[:lo]))
    return before, before + int(np.count_nonzero(flags[lo:hi]))


def slab_tables(t: dict, z0: int, z1: int) -> dict:
    """The setup tables of cell planes [z0, z1) (0-based) of a global mesh,
    as a mesh of its own: special cells, PML cells, excitation and output
    cells keep their traversal order and are renumbered from 1; the
    parameter, material and excitation-function tables are shared.
    ``slab`` = (a slab below, a slab above); the outer boundary is not
    applied on those sides (their ghost planes are filled by the exchange).
    ``slab_points`` lists the global indices of the centre output points
    the slab holds (in its own output order), ``slab_z0`` its first plane."""
    check_shardable(t)
    nx, ny, nz = int(t["nx"]), int(t["ny"]), int(t["nz"])
    if not 0 <= z0 < z1 <= nz:
        raise ValueError("slab outside the mesh")
    plane = nx * ny
    code = np.asarray(t["cell_code"]).reshape(-1)
    is_sp = code != 0
    sa, sb = _range_of(is_sp, z0 * plane, z1 * plane)
    s = dict(t)
    s["nz"] = z1 - z0
    c = code[z0 * plane: z1 * plane].astype(np.int32)
    s["cell_code"] = np.where(c != 0, c - sa, 0).astype(np.int32)
    s["n_special"] = sb - sa
    for k in ("sp_material", "sp_excitation", "sp_output"):
        s[k] = np.asarray(t[k])[sa:sb].copy()
    # PML numbers: traversal order over the PML cells
    sp_pml_g = np.asarray(t["sp_pml"])
    pa = int(np.count_nonzero(sp_pml_g[:sa]))
    pml = sp_pml_g[sa:sb]
    s["sp_pml"] = np.where(pml != 0, pml - pa, 0).astype(np.int32)
    npml = int(np.count_nonzero(pml))
    s["n_pml_cells"] = npml
    s["pml_cell_param"] = np.asarray(t["pml_cell_param"])[pa:pa + npml].copy()
    s["n_pml_material_cells"] = int(np.count_nonzero((pml != 0) & (s["sp_material"] != 0)))
    # excitation cells (numbered in traversal order) and the point sources in the slab
    exc_g = np.asarray(t["sp_excitation"]) != 0
    ea = int(np.count_nonzero(exc_g[:sa]))
    ne = int(np.count_nonzero(exc_g[sa:sb]))
    s["n_exc_cells"] = ne
    pt_cell = np.asarray(t["pt_cell"])
    keep_pt = (pt_cell > ea) & (pt_cell <= ea + ne)
    s["pt_cell"] = (pt_cell[keep_pt] - ea).astype(np.int32)
    for k in ("pt_comp", "pt_fn", "pt_type"):
        s[k] = np.asarray(t[k])[keep_pt].copy()
    s["n_exc_points"] = int(keep_pt.sum())
    if "pt_xyz" in t:
        s["pt_xyz"] = _shift_z(np.asarray(t["pt_xyz"]).reshape(-1, 3)[keep_pt], z0)
    # output cells and the centre output points in the slab
    out_g = np.asarray(t["sp_output"]) != 0
    oa = int(np.count_nonzero(out_g[:sa]))
    no = int(np.count_nonzero(out_g[sa:sb]))
    s["n_out_cells"] = no
    out_cell = np.asarray(t["out_cell"])
    keep_o = (out_cell > oa) & (out_cell <= oa + no)
    s["out_cell"] = (out_cell[keep_o] - oa).astype(np.int32)
    s["out_comp"] = np.asarray(t["out_comp"])[keep_o].copy()
    if "out_keep" in t:
        s["out_keep"] = np.asarray(t["out_keep"])[oa:oa + no].copy()
    if "out_point_no" in t:
        s["out_point_no"] = np.asarray(t["out_point_no"])[keep_o].copy()
    if "out_xyz" in t:
        s["out_xyz"] = _shift_z(np.asarray(t["out_xyz"]).reshape(-1, 3)[keep_o], z0)
    s["slab_points"] = np.nonzero(keep_o)[0].astype(np.int32)
    below, above = z0 > 0, z1 < nz
    s["slab"] = np.array([int(below), int(above)], dtype=np.int32)
    s["slab_z0"] = z0
    _slab_faces(t, s, z0, z1)
    if "pml_depth" in t:
        d = np.asarray(t["pml_depth"]).copy()
        d[4] = max(0, int(d[4]) - z0) if not below else 0
        d[5] = max(0, int(d[5]) - (nz - z1)) if not above else 0
        s["pml_depth"] = d
    return s


def _slab_faces(t: dict, s: dict, z0: int, z1: int) -> None:
    """The special faces of planes [z0, z1) (connect.F90 order: cz, cy, cx,
    then the x-, y-, z-face, so a slab's faces are one run of the list, and
    so are its excitation and output face numbers), with the sources,
    probes, sheets and frequency output surface entries on them renumbered.
    ``slab_face_probes`` and ``slab_dft`` give the global positions of the
    slab's face probes and DFT faces, for the gathers."""
    n = int(t.get("n_faces", 0))
    cz = np.asarray(t.get("face_cz", []), dtype=np.int64)
    fdir = np.asarray(t.get("face_dir", []), dtype=np.int64)
    keep = (cz > z0) & (cz <= z1)
    if n and np.any(keep & (fdir == 3) & (cz == z0 + 1) & (z0 > 0)):
        raise UnsupportedFeature("z-slab sharding with a special face on the z-faces between two slabs")
    fe = np.asarray(t.get("face_exc", []), dtype=np.int64)
    fo = np.asarray(t.get("face_out", []), dtype=np.int64)
    ea = int(np.count_nonzero(fe[~keep & (cz <= z0)])) if n else 0
    oa = int(np.count_nonzero(fo[~keep & (cz <= z0)])) if n else 0
    ne, no = (int(np.count_nonzero(fe[keep])), int(np.count_nonzero(fo[keep]))) if n else (0, 0)
    s["n_faces"] = int(np.count_nonzero(keep))
    for k in ("face_cx", "face_cy", "face_dir", "face_mat", "face_smat"):
        if k in t:
            s[k] = np.asarray(t[k])[keep].astype(np.int32) if n else np.asarray(t[k]).copy()
    s["face_cz"] = (cz[keep] - z0).astype(np.int32)
    s["face_exc"] = np.where(fe[keep] != 0, fe[keep] - ea, 0).astype(np.int32)
    s["face_out"] = np.where(fo[keep] != 0, fo[keep] - oa, 0).astype(np.int32)
    s["n_exc_faces"], s["n_out_faces"] = ne, no

    def in_exc(a):
        a = np.asarray(a, dtype=np.int64)
        return (a > ea) & (a <= ea + ne)

    def in_out(a):
        a = np.asarray(a, dtype=np.int64)
        return (a > oa) & (a <= oa + no)

    # Huygens patches (their offsets stay the global ones)
    hk = in_exc(t.get("hs_face_exc", []))
    if int(t.get("hs_n", 0)):
        s["hs_face_exc"] = (np.asarray(t["hs_face_exc"])[hk] - ea).astype(np.int32)
        s["hs_norm"] = np.asarray(t["hs_norm"]).reshape(-1, 3)[hk].reshape(-1).astype(np.int32)
        s["hs_offset"] = np.asarray(t["hs_offset"])[hk].copy()
        s["hs_n"] = int(hk.sum())
    # face sources
    pk = in_exc(t.get("fpt_face", []))
    s["fpt_face"] = (np.asarray(t.get("fpt_face", []), dtype=np.int64)[pk] - ea).astype(np.int32)
    for k in ("fpt_comp", "fpt_fn", "fpt_type", "fpt_side", "fpt_scale"):
        if k in t:
            s[k] = np.asarray(t[k])[pk].copy()
    s["n_face_points"] = int(pk.sum())
    # face probes
    qk = in_out(t.get("fprobe_face", []))
    s["fprobe_face"] = (np.asarray(t.get("fprobe_face", []), dtype=np.int64)[qk] - oa).astype(np.int32)
    for k in ("fprobe_side", "fprobe_comp", "fprobe_point_no"):
        if k in t:
            s[k] = np.asarray(t[k])[qk].copy()
    s["n_face_probes"] = int(qk.sum())
    s["slab_face_probes"] = np.nonzero(qk)[0].astype(np.int32)
    # frequency output surfaces: every entry, with the slab's faces of each
    if int(t.get("n_dft", 0)):
        ptr = np.asarray(t["dft_face_ptr"], dtype=np.int64)
        dk = in_out(t["dft_face_out"])
        s["dft_face_out"] = (np.asarray(t["dft_face_out"], dtype=np.int64)[dk] - oa).astype(np.int32)
        s["dft_face_side"] = np.asarray(t["dft_face_side"])[dk].copy()
        s["dft_face_ptr"] = np.array([int(np.count_nonzero(dk[:p])) for p in ptr], dtype=np.int32)
        s["slab_dft"] = np.nonzero(dk)[0].astype(np.int32)
    else:
        s["slab_dft"] = np.zeros(0, dtype=np.int32)


def gather_rows(n_rows: int, slabs: List[dict], key: str, parts: List[np.ndarray]) -> np.ndarray:
    """Global rows (face probe series, DFT phasors) from each slab's rows,
    placed by the slab's ``key`` positions."""
    shape = next((np.asarray(p).shape[1:] for p in parts if np.asarray(p).size), ())
    out = np.zeros((n_rows,) + tuple(shape))
    for tab, rows in zip(slabs, parts):
        for k, g in enumerate(np.asarray(tab[key])):
            out[int(g)] = rows[k]
    return out


def _shift_z(xyz: np.ndarray, z0: int) -> np.ndarray:
    out = np.asarray(xyz, dtype=np.int32).copy().reshape(-1, 3)
    out[:, 2] -= z0
    return out


def split(t: dict, parts: int) -> List[dict]:
    """The slab tables of every part of ``slab_bounds(nz, parts)``."""
    return [slab_tables(t, z0, z1) for z0, z1 in slab_bounds(int(t["nz"]), parts)]


def gather_series(t: dict, slabs: List[dict], series: List[np.ndarray]) -> np.ndarray:
    """Probe series [n_points, steps] of the global mesh from each slab's
    ``probe_series``."""
    n_pts = len(np.asarray(t["out_cell"]))
    steps = max((s.shape[1] for s in series if s.size), default=0)
    out = np.zeros((n_pts, steps))
    for tab, ser in zip(slabs, series):
        for k, g in enumerate(np.asarray(tab["slab_points"])):
            out[int(g)] = ser[k]
    return out


class GpuSlab:
    """One slab on a GPU behind the stepping interface the exchange uses
    (``run``, ``halo_bytes``, ``halo_get`` / ``halo_put`` into device
    tensors)."""

    def __init__(self, tables: dict, precision: int, device: int = 0):
        from . import capi

        self.t = tables
        self.device = device
        self.mesh = capi.GpuMesh(tables, precision=precision, device=device)

    def run(self, n: int):
        self.mesh.run(n, sync=False)

    def halo_bytes(self) -> int:
        return self.mesh.halo_bytes()

    def halo_get(self, side: int, buf):
        self.mesh.halo_get(side, buf.data_ptr())

    def halo_put(self, side: int, buf):
        self.mesh.halo_put(side, buf.data_ptr())

    def probes(self) -> np.ndarray:
        from .problem import probe_series

        self.mesh.synchronize()
        return probe_series(self.t, self.mesh.cell_output())

    def face_probes(self) -> np.ndarray:
        self.mesh.synchronize()
        return self.mesh.face_output()

    def dft(self) -> np.ndarray:
        self.mesh.synchronize()
        return self.mesh.dft()

    def close(self):
        self.mesh.close()


class LocalShards:
    """All slabs of one mesh in this process (on one GPU, or one per device
    of ``devices``), the halos exchanged by device-to-device copies between
    timesteps.  Results are those of the unpartitioned mesh."""

    def __init__(self, t: dict, parts: int, precision: int, devices=None, slab_factory=None):
        import torch

        self.t = t
        self.tables = split(t, parts)
        devices = list(devices) if devices is not None else [0] * parts
        make = slab_factory or (lambda tab, dev: GpuSlab(tab, precision, dev))
        self.slabs = [make(tab, devices[i]) for i, tab in enumerate(self.tables)]
        nb = self.slabs[0].halo_bytes()
        self.up = [torch.empty(nb, dtype=torch.uint8, device=f"cuda:{devices[i]}") for i in range(parts - 1)]
        self.down = [torch.empty(nb, dtype=torch.uint8, device=f"cuda:{devices[i + 1]}") for i in range(parts - 1)]

    def exchange(self):
        for i in range(len(self.slabs) - 1):
            lo, hi = self.slabs[i], self.slabs[i + 1]
            lo.halo_get(1, self.up[i])
            hi.halo_put(0, self.up[i])
            hi.halo_get(0, self.down[i])
            lo.halo_put(1, self.down[i])

    def run(self, n: int):
        for _ in range(n):
            for s in self.slabs:
                s.run(1)
            self.exchange()

    def probes(self) -> np.ndarray:
        return gather_series(self.t, self.tables, [s.probes() for s in self.slabs])

    def face_probes(self) -> np.ndarray:
        """Face probe series [n_face_probes, steps] of the global mesh."""
        return gather_rows(int(self.t.get("n_face_probes", 0)), self.tables, "slab_face_probes",
                           [s.face_probes() for s in self.slabs])

    def dft(self) -> np.ndarray:
        """Frequency output surface phasors [faces, 2] in the global entry order."""
        n = int(np.asarray(self.t["dft_face_ptr"])[-1]) if int(self.t.get("n_dft", 0)) else 0
        return gather_rows(n, self.tables, "slab_dft", [s.dft() for s in self.slabs])

    def close(self):
        for s in self.slabs:
            s.close()


class DistShard:
    """This rank's slab of a mesh partitioned over the ranks of
    ``torch.distributed`` (rank r holds slab r of ``slab_bounds``), with the
    halos exchanged point-to-point with the neighbour ranks between
    timesteps (``batch_isend_irecv``: NCCL over NVLink on GPUs).  Every rank
    takes the same steps; ``probes`` gathers the global probe series on
    rank 0 (``None`` elsewhere)."""

    def __init__(self, t: dict, precision: int = None, device: int = 0, slab_factory=None, group=None):
        import torch
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.t = t
        z0, z1 = slab_bounds(int(t["nz"]), self.world)[self.rank]
        self.tab = slab_tables(t, z0, z1)
        make = slab_factory or (lambda tab, dev: GpuSlab(tab, precision, dev))
        self.slab = make(self.tab, device)
        nb = self.slab.halo_bytes()
        dev = torch.device(f"cuda:{device}") if dist.get_backend(group) == "nccl" else torch.device("cpu")
        if dev.type == "cuda":  # NCCL point-to-point needs the rank's device current
            torch.cuda.set_device(dev)
        self.bufs = {k: torch.empty(nb, dtype=torch.uint8, device=dev) for k in ("send_up", "send_dn", "recv_up",
                                                                                  "recv_dn")}
        self.on_gpu = dev.type == "cuda"

    def _peer(self, r: int) -> int:
        return r if self.group is None else self.dist.get_global_rank(self.group, r)

    def exchange(self):
        import torch

        d, b, r, w = self.dist, self.bufs, self.rank, self.world
        ops = []
        if r + 1 < w:
            self.slab.halo_get(1, b["send_up"])
            ops += [d.P2POp(d.isend, b["send_up"], self._peer(r + 1), self.group),
                    d.P2POp(d.irecv, b["recv_up"], self._peer(r + 1), self.group)]
        if r > 0:
            self.slab.halo_get(0, b["send_dn"])
            ops += [d.P2POp(d.isend, b["send_dn"], self._peer(r - 1), self.group),
                    d.P2POp(d.irecv, b["recv_dn"], self._peer(r - 1), self.group)]
        if ops:
            for q in d.batch_isend_irecv(ops):
                q.wait()
        if self.on_gpu:
            torch.cuda.current_stream().synchronize()
        if r + 1 < w:
            self.slab.halo_put(1, b["recv_up"])
        if r > 0:
            self.slab.halo_put(0, b["recv_dn"])

    def run(self, n: int):
        for _ in range(n):
            self.slab.run(1)
            self.exchange()

    def probes(self):
        """Global probe series on rank 0 (gathered over the ranks), None elsewhere."""
        mine = self.slab.probes()
        parts = [None] * self.world if self.rank == 0 else None
        self.dist.gather_object((self.tab["slab_points"].tolist(), mine), parts, dst=self._peer(0), group=self.group)
        if self.rank != 0:
            return None
        n_pts = len(np.asarray(self.t["out_cell"]))
        steps = max((p[1].shape[1] for p in parts if p[1].size), default=0)
        out = np.zeros((n_pts, steps))
        for pts, ser in parts:
            for k, g in enumerate(pts):
                out[int(g)] = ser[k]
        return out

    def _gather(self, key: str, rows: np.ndarray, n_rows: int):
        parts = [None] * self.world if self.rank == 0 else None
        self.dist.gather_object((self.tab[key].tolist(), rows), parts, dst=self._peer(0), group=self.group)
        if self.rank != 0:
            return None
        return gather_rows(n_rows, [{key: p[0]} for p in parts], key, [p[1] for p in parts])

    def face_probes(self):
        """Global face probe series on rank 0, None elsewhere."""
        return self._gather("slab_face_probes", self.slab.face_probes(), int(self.t.get("n_face_probes", 0)))

    def dft(self):
        """Global frequency output surface phasors on rank 0, None elsewhere."""
        n = int(np.asarray(self.t["dft_face_ptr"])[-1]) if int(self.t.get("n_dft", 0)) else 0
        return self._gather("slab_dft", self.slab.dft(), n)

    def close(self):
        self.slab.close()
