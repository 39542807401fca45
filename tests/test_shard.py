"""z-slab partitioning (ggi_tlm_b200/shard.py), the replacement for the
reference's MPI build (mesh_partition, MESH/general_mesh_subroutines.F90:868-972;
TLM_parallel_pass_data_1/2, TLM_SOLVER/TLM_parallel_pass_data.F90:38-279).

CPU: the slab tables against the global ones; the oracle's slab mode
(the reference's two passes a step) run slab by slab, serially and as two
gloo ranks, gives the unpartitioned oracle's probe series bit for bit, with
special faces too (a Huygens plane or a Huygens box cut by the slab
boundaries, face sources, face probes, a frequency output surface); the
exchange wiring and the gathers of DistShard over gloo ranks.  GPU: every
slab of a mesh on one GPU (LocalShards, halos by device copies between
steps) against the unpartitioned GPU run (bit-identical) and the oracle."""
import os
import socket
import sys

import numpy as np
import pytest

from ggi_tlm_b200 import cases, shard
from ggi_tlm_b200.problem import (Block, OutputPoint, PointExcitation, UnsupportedFeature, VolumeMaterial, build_tables,
                                  probe_series)

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)
import oracle  # noqa: E402


def spec(nx=18, ny=14, nz=23, steps=60):
    """A PML box with a dielectric block that straddles slab boundaries, a
    point source and probes on several planes."""
    s = cases.pml_point_source(nx, ny, nz, pml=3, steps=steps, dl=0.01, n_probes=0)
    s.materials = [VolumeMaterial.dielectric(3.0, 0.2)]
    s.material_regions = [(1, Block(6, 12, 5, 10, 9, 16))]
    s.outputs = [OutputPoint((9, 7, z), "Ex") for z in (2, 8, 11, 12, 16, 21)] + [OutputPoint((5, 6, 12), "Hz")]
    return s


def test_slab_bounds_follow_mesh_partition():
    for nz, parts in ((23, 2), (23, 3), (64, 8), (7, 7)):
        b = shard.slab_bounds(nz, parts)
        owner = [int(parts * (cz - 1) / nz) for cz in range(1, nz + 1)]
        for r, (z0, z1) in enumerate(b):
            assert all(owner[z] == r for z in range(z0, z1))
        assert b[0][0] == 0 and b[-1][1] == nz and all(b[i][1] == b[i + 1][0] for i in range(parts - 1))
    with pytest.raises(ValueError):
        shard.slab_bounds(4, 5)


def test_slab_tables_cover_the_mesh():
    t = build_tables(spec())
    parts = shard.split(t, 3)
    assert sum(p["nz"] for p in parts) == t["nz"]
    assert sum(p["n_special"] for p in parts) == t["n_special"]
    assert sum(p["n_pml_cells"] for p in parts) == t["n_pml_cells"]
    np.testing.assert_array_equal(np.concatenate([p["pml_cell_param"] for p in parts]), t["pml_cell_param"])
    np.testing.assert_array_equal(np.concatenate([p["sp_material"] for p in parts]), t["sp_material"])
    assert sorted(np.concatenate([p["slab_points"] for p in parts]).tolist()) == list(range(len(t["out_cell"])))
    assert sum(p["n_exc_points"] for p in parts) == t["n_exc_points"]
    codes = np.concatenate([np.where(p["cell_code"] > 0, p["cell_code"] + off, 0)
                            for p, off in zip(parts, np.cumsum([0] + [p["n_special"] for p in parts[:-1]]))])
    np.testing.assert_array_equal(codes, t["cell_code"])
    assert [tuple(p["slab"]) for p in parts] == [(0, 1), (1, 1), (1, 0)]


def face_spec(steps=60):
    """A PML box with dielectric spheres, a Huygens plane wave, a frequency
    output surface, face sources and face probes on several planes."""
    s = cases.pml_spheres(n=26, pml=3, n_spheres=2, steps=steps, n_probes=3, n_freq=2, dft_size=6, rmin=2.0,
                          rmax=3.0)
    s.point_excitations.append(PointExcitation((9, 10, 20), "Ex", 1, face="zmin"))
    s.point_excitations.append(PointExcitation((12, 8, 7), "Hy", 1, face="xmax", one_side=True, scale=0.5))
    s.outputs += [OutputPoint((13, 13, 18), "Ey", face="ymax"), OutputPoint((10, 9, 6), "Hx", face="zmin")]
    return s


def test_whole_surface_outputs_and_slab_boundary_faces_are_refused():
    t = build_tables(face_spec())
    t2 = dict(t, n_ff=1)
    with pytest.raises(UnsupportedFeature, match="sharding"):
        shard.split(t2, 2)
    # the z-face source at cz = 20 lies between planes 19 and 20: the boundary of 2 slabs of 23 + 3 planes?
    z = [b for b in shard.slab_bounds(int(t["nz"]), 4)]
    cut = z[1][0]  # first plane (0-based) of slab 1
    s = face_spec()
    s.point_excitations.append(PointExcitation((9, 10, cut + 1), "Ex", 1, face="zmin"))
    with pytest.raises(UnsupportedFeature, match="between two slabs"):
        shard.split(build_tables(s), 4)


def test_slab_faces_partition_the_faces():
    t = build_tables(face_spec())
    parts = shard.split(t, 3)
    assert sum(p["n_faces"] for p in parts) == int(t["n_faces"])
    assert sum(p["hs_n"] for p in parts) == int(t["hs_n"])
    assert sum(p["n_face_points"] for p in parts) == int(t["n_face_points"])
    assert sorted(g for p in parts for g in p["slab_face_probes"]) == list(range(int(t["n_face_probes"])))
    assert sorted(g for p in parts for g in p["slab_dft"]) == list(range(int(t["dft_face_ptr"][-1])))


def run_oracle_slabs(t, parts, extras=False):
    """The reference's partitioned step on the oracle, every slab in this
    process: scatter, pass 1 (top plane up), connect, pass 2 (back down).
    With ``extras`` also the gathered face probes and DFT phasors."""
    tabs = shard.split(t, parts)
    os_ = [oracle.Oracle(s) for s in tabs]
    rows = [[] for _ in tabs]
    for _ in range(int(t["n_timesteps"])):
        for k, o in enumerate(os_):
            rows[k].append(o.half_step(1))
        for k in range(parts - 1):  # TLM_parallel_pass_data_1
            os_[k + 1].set_zplane(0, os_[k].zplane(1))
        for o in os_:
            o.half_step(2)
        for k in range(parts - 1):  # TLM_parallel_pass_data_2
            os_[k].set_zplane(1, os_[k + 1].zplane(0))
    series = [probe_series(s, np.array(r)) for s, r in zip(tabs, rows)]
    fp = [o.face_probes() if int(s["n_face_probes"]) else np.zeros((0, 0)) for o, s in zip(os_, tabs)]
    dft = [o.dft() for o in os_] if int(t.get("n_dft", 0)) else []
    for o in os_:
        o.close()
    got = shard.gather_series(t, tabs, series)
    if not extras:
        return got
    n_dft = int(t["dft_face_ptr"][-1]) if int(t.get("n_dft", 0)) else 0
    return (got, shard.gather_rows(int(t["n_face_probes"]), tabs, "slab_face_probes", fp),
            shard.gather_rows(n_dft, tabs, "slab_dft", dft))


@pytest.mark.parametrize("parts", [2, 3])
def test_oracle_slabs_with_special_faces_match_the_unpartitioned_oracle(parts):
    t = build_tables(face_spec())
    o = oracle.Oracle(t)
    want = probe_series(t, o.run(int(t["n_timesteps"])))
    want_fp, want_dft = o.face_probes(), o.dft()
    got, fp, dft = run_oracle_slabs(t, parts, extras=True)
    np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(fp, want_fp)
    np.testing.assert_array_equal(dft, want_dft)
    assert np.abs(want_fp).max() > 0 and np.abs(want_dft).max() > 0


@pytest.mark.parametrize("parts", [2, 3, 5])
def test_oracle_slabs_match_the_unpartitioned_oracle(parts):
    t = build_tables(spec())
    want = probe_series(t, oracle.Oracle(t).run(int(t["n_timesteps"])))
    got = run_oracle_slabs(t, parts)
    np.testing.assert_array_equal(got, want)
    assert np.abs(want).max() > 0


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_rank(rank, world, port, q):
    """One gloo rank: its slab on the oracle, the two passes over gloo."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch
    import torch.distributed as dist
    import oracle as orc
    from ggi_tlm_b200 import shard as sh
    from ggi_tlm_b200.problem import build_tables as bt, probe_series as ps

    dist.init_process_group("gloo", rank=rank, world_size=world)
    t = bt(spec())
    z0, z1 = sh.slab_bounds(int(t["nz"]), world)[rank]
    tab = sh.slab_tables(t, z0, z1)
    o = orc.Oracle(tab)
    shape = (2, int(t["ny"]), int(t["nx"]))
    rows = []
    for _ in range(int(t["n_timesteps"])):
        rows.append(o.half_step(1))
        if rank + 1 < world:
            dist.send(torch.from_numpy(o.zplane(1)), rank + 1)
        if rank > 0:
            buf = torch.zeros(shape, dtype=torch.float64)
            dist.recv(buf, rank - 1)
            o.set_zplane(0, buf.numpy())
        o.half_step(2)
        if rank > 0:
            dist.send(torch.from_numpy(o.zplane(0)), rank - 1)
        if rank + 1 < world:
            buf = torch.zeros(shape, dtype=torch.float64)
            dist.recv(buf, rank + 1)
            o.set_zplane(1, buf.numpy())
    q.put((rank, tab["slab_points"].tolist(), ps(tab, np.array(rows))))
    o.close()
    dist.destroy_process_group()


def test_oracle_slabs_over_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps_ = [ctx.Process(target=_oracle_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps_:
        p.start()
    res = [q.get(timeout=300) for _ in range(2)]
    for p in ps_:
        p.join(60)
        assert p.exitcode == 0
    t = build_tables(spec())
    want = probe_series(t, oracle.Oracle(t).run(int(t["n_timesteps"])))
    got = np.zeros_like(want)
    for _, pts, ser in res:
        for k, g in enumerate(pts):
            got[g] = ser[k]
    np.testing.assert_array_equal(got, want)


class FakeSlab:
    """Stands in for a GPU slab: each halo it sends encodes (rank, step,
    side); each halo it receives must come from the right neighbour, step
    and side."""

    def __init__(self, tab, rank, world):
        self.t, self.rank, self.world, self.step, self.seen = tab, rank, world, 0, []

    def run(self, n):
        self.step += n

    def halo_bytes(self):
        return 24

    def halo_get(self, side, buf):
        import torch

        buf.view(torch.float64)[:] = torch.tensor([self.rank, self.step, side], dtype=torch.float64)

    def halo_put(self, side, buf):
        import torch

        v = buf.view(torch.float64).tolist()
        want = [self.rank - 1, self.step, 1] if side == 0 else [self.rank + 1, self.step, 0]
        assert v == want, (self.rank, side, v, want)
        self.seen.append((self.step, side))

    def probes(self):
        n = len(self.t["out_cell"])
        return np.full((n, 1), float(self.rank))

    def face_probes(self):
        return np.full((int(self.t["n_face_probes"]), 1), float(self.rank))

    def dft(self):
        return np.full((int(self.t["dft_face_ptr"][-1]), 2), float(self.rank))

    def close(self):
        pass


def _fake_rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from ggi_tlm_b200 import shard as sh
    from ggi_tlm_b200.problem import build_tables as bt

    dist.init_process_group("gloo", rank=rank, world_size=world)
    t = bt(face_spec())
    ds = sh.DistShard(t, slab_factory=lambda tab, dev: FakeSlab(tab, rank, world))
    ds.run(5)
    seen = ds.slab.seen
    pr, fp, dft = ds.probes(), ds.face_probes(), ds.dft()
    q.put((rank, seen, None if pr is None else pr.tolist(), None if fp is None else fp[:, 0].tolist(),
           None if dft is None else dft[:, 0].tolist()))
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_dist_shard_exchange_wiring_over_gloo(world):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps_ = [ctx.Process(target=_fake_rank, args=(r, world, port, q)) for r in range(world)]
    for p in ps_:
        p.start()
    res = {r: (seen, pr, fp, dft) for r, seen, pr, fp, dft in (q.get(timeout=120) for _ in range(world))}
    for p in ps_:
        p.join(60)
        assert p.exitcode == 0
    for r in range(world):
        sides = ([1] if r + 1 < world else []) + ([0] if r > 0 else [])
        assert sorted(res[r][0]) == sorted((s, d) for s in range(1, 6) for d in sides)
    t = build_tables(face_spec())
    owner, fowner, downer = {}, {}, {}
    for r, (z0, z1) in enumerate(shard.slab_bounds(int(t["nz"]), world)):
        tab = shard.slab_tables(t, z0, z1)
        owner.update({int(g): r for g in tab["slab_points"]})
        fowner.update({int(g): r for g in tab["slab_face_probes"]})
        downer.update({int(g): r for g in tab["slab_dft"]})
    assert [row[0] for row in res[0][1]] == [float(owner[g]) for g in range(len(t["out_cell"]))]
    # face probes and DFT phasors gathered on rank 0 in global order, from the ranks that hold them
    assert res[0][2] == [float(fowner[g]) for g in range(int(t["n_face_probes"]))]
    assert res[0][3] == [float(downer[g]) for g in range(int(t["dft_face_ptr"][-1]))]
    assert len(set(downer.values())) >= 1 and all(res[r][1] is None for r in range(1, world))


@pytest.mark.gpu
@pytest.mark.parametrize("parts", [2, 3])
def test_gpu_slabs_match_the_unpartitioned_mesh(gpu_lib, parts):
    from ggi_tlm_b200 import capi

    t = build_tables(spec(steps=80))
    want64 = probe_series(t, oracle.Oracle(t).run(int(t["n_timesteps"])))
    for prec in (capi.TLM_PRECISION_FP64, capi.TLM_PRECISION_FP32):
        with capi.GpuMesh(t, precision=prec) as g:
            g.run(int(t["n_timesteps"]))
            whole = probe_series(t, g.cell_output())
        ls = shard.LocalShards(t, parts, prec)
        ls.run(int(t["n_timesteps"]))
        got = ls.probes()
        ls.close()
        np.testing.assert_array_equal(got, whole)
        if prec == capi.TLM_PRECISION_FP64:
            assert np.linalg.norm(got - want64) <= 1e-10 * np.linalg.norm(want64)


@pytest.mark.parametrize("parts", [3, 5])
def test_oracle_slabs_cut_through_a_huygens_box(parts):
    """HUYGENS_SURFACE (40^3, a Huygens box of 20^3 cells): the slab
    boundaries cut the box's x- and y-faces, whose patches go to the slab
    that holds their plane (its output surfaces and volumes left out)."""
    import test_inp

    from ggi_tlm_b200 import inp

    spec = inp.read_inp(test_inp.inputs()["huygens_box"], test_inp.materials).spec
    spec.output_surfaces, spec.output_volumes = [], []  # whole-surface outputs: not sharded
    t = build_tables(spec)
    with pytest.raises(UnsupportedFeature, match="between two slabs"):
        shard.split(t, 2)  # the face probes on the z-faces of cell plane 21 lie on the cut
    tabs = shard.split(t, parts)
    assert sum(1 for p in tabs if p["hs_n"]) >= 2
    want = probe_series(t, oracle.Oracle(t).run(int(t["n_timesteps"])))
    np.testing.assert_array_equal(run_oracle_slabs(t, parts), want)


@pytest.mark.gpu
@pytest.mark.parametrize("parts", [2, 3])
def test_gpu_slabs_with_special_faces_match_the_unpartitioned_mesh(gpu_lib, parts):
    """The Huygens plane, the frequency output surface, face sources and
    face probes split over slabs on one GPU: probes, face probes and DFT
    phasors bit-identical to the unpartitioned GPU run, and within 1e-10
    of the oracle in FP64."""
    from ggi_tlm_b200 import capi

    t = build_tables(face_spec(steps=80))
    n = int(t["n_timesteps"])
    o = oracle.Oracle(t)
    want64 = probe_series(t, o.run(n))
    want_dft = o.dft()
    for prec in (capi.TLM_PRECISION_FP64, capi.TLM_PRECISION_FP32):
        with capi.GpuMesh(t, precision=prec) as g:
            g.run(n)
            whole, whole_fp, whole_dft = probe_series(t, g.cell_output()), g.face_output(), g.dft()
        ls = shard.LocalShards(t, parts, prec)
        ls.run(n)
        got, fp, dft = ls.probes(), ls.face_probes(), ls.dft()
        ls.close()
        np.testing.assert_array_equal(got, whole)
        np.testing.assert_array_equal(fp, whole_fp)
        np.testing.assert_array_equal(dft, whole_dft)
        if prec == capi.TLM_PRECISION_FP64:
            assert np.linalg.norm(got - want64) <= 1e-10 * np.linalg.norm(want64)
            assert np.linalg.norm(dft - want_dft) <= 1e-10 * np.linalg.norm(want_dft)
