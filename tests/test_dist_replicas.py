"""The N>1 host path of bench.py on CPU: world_size-2 gloo ranks.

bench.py runs N independent replicas (the solve does not shard); what
crosses ranks is a barrier around the timed region and a max-reduction of
the per-rank device time.  These tests run that plumbing as two gloo ranks,
and the reference arm under torchrun, where rank 0 alone must print one
JSON line and the other rank must exit 0 without work.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist

    w, r, _ = bench.dist_setup()
    assert (w, r) == (world, rank)
    assert dist.get_backend() == "gloo"
    bench.barrier(w)
    local_ms = 100.0 + 50.0 * r  # rank 1 is the slow one
    value, ms = bench.replica_rate(1000, 10, w, local_ms)
    bench.barrier(w)
    dist.destroy_process_group()
    q.put((r, value, ms))


def test_replica_rate_is_max_over_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=5) for _ in range(2))
    for _, value, ms in res:
        assert ms == 150.0  # every rank sees the slowest rank's time
        assert value == pytest.approx(1000 * 10 * 2 / 0.150 / 1e9)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    value, ms = bench.replica_rate(1000, 10, 1, 100.0)
    assert ms == 100.0 and value == pytest.approx(1e-4)


def test_reference_arm_under_torchrun_prints_once_from_rank_0():
    env = dict(os.environ, TLM_REFERENCE_BUDGET_S="1", CUDA_VISIBLE_DEVICES="")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "2",
           "--warmup", "0", "--workload", "c1"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port"
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
