#!/usr/bin/env python
"""Benchmark of the B200 SCN-TLM time-stepping core.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload t512|t192|c2|c3|c1]

One "step" is one TLM time step (excitation, scatter, connect, outer boundary,
probes) over the whole mesh.  Default workload: the 512^3 free-space box with
an 8-cell PML on all six faces, a Gaussian point source and 4 probes (seeded
synthetic input, 2000 steps).  The headline ``value`` is the plain FP64 path,
the reference's own precision; the FP32 fast path (FP32 links, FP64 filter,
PML recursion and DFT) and its probe error over the complete solve are in
the ``fp32`` key.  The metric is cell-updates per second (whole job, all
GPUs), with the bulk cell kernel's achieved HBM bandwidth against the
measured copy peak.  Sections at N=1: the 256^3 PML-spheres mesh (c2), the
384x384x192 Debye-slab mesh (c3), 96 uneven boxes batched (c4) and the
serving trace (c5).

Multi-GPU (torchrun, one process per GPU): the path does not shard here
(replicas only); every rank advances its own copy of the mesh, the timed
region is bracketed by barriers and the time is the max over ranks.

``--impl reference`` times the reference's CPU path on the host cores: the
oracle's C restatement of the reference's sequential loop (the Fortran
builds cannot be compiled on this box), z-planes shared among all host
threads, on the same tables.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gcell-updates/s & %HBM roofline (FP32 vs FP64, 1 B200); serving solves/s, p50/p99"
UNIT = "Gcell-updates/s"
FALLBACK_HBM_GBS = 6650.0


# Bulk (free-space) cell-kernel configurations of the library, by variant
# index: (cells per tile, staging depth) for FP32 and FP64; 0 = the
# register-pipelined kernel without TMA staging.
BULK_VARIANTS = [(0, 0, 0, 0), (1024, 2, 512, 2), (512, 3, 256, 3), (512, 4, 256, 4), (1024, 3, 512, 3),
                 (256, 6, 128, 6)]

# DRAM traffic of the bulk kernel (dram__bytes_read.sum + dram__bytes_write.sum)
# per free-space cell it updates, from one ncu capture of the FP64 kernel; the
# traffic of a launch grows with the cells it updates, so a full launch is
# this figure times its cells.
NCU_TRAFFIC = {
    "pml_point_source_512^3_pml8": {
        "bytes_per_cell": 194.95,
        "source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one tlm_bulk_tma_kernel<double,2,512,2> "
                  "launch on the same mesh at 192^3 (1062.8 MB for 5 451 771 free-space cells, "
                  "profiles/tlm_bulk_tma_kernel_pml_point_source_192_fp64.md), scaled to 512^3 by the free-space "
                  "cell count"},
}


def bulk_kernel_name(variant: int, vec: int) -> str:
    t32, s32, t64, s64 = BULK_VARIANTS[variant]
    if variant == 0:
        return f"tlm_cell_kernel<{'float' if vec == 4 else 'double'},{vec}>"
    tile, st = (t32, s32) if vec == 4 else (t64, s64)
    return f"tlm_bulk_tma_kernel<{'float' if vec == 4 else 'double'},{vec},{tile},{st}>"


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def workload_spec(name: str):
    from ggi_tlm_b200 import cases

    if name == "c2":
        return cases.pml_spheres(), "pml_spheres_256^3_pml8_32spheres_huygens_dft64x64x64"
    if name == "t512":
        return cases.pml_point_source(512, steps=2000), "pml_point_source_512^3_pml8"
    if name == "t192":  # the same mesh at 192^3: small enough for an ncu capture
        return cases.pml_point_source(192, steps=300), "pml_point_source_192^3_pml8"
    if name == "c3":
        return cases.debye_slabs(), "debye_slabs_384x384x192_pml10_6slabs_dft64x64x64"
    if name == "c3h":  # the same configuration at half the edge lengths: small enough for an ncu capture
        return (cases.debye_slabs(192, 192, 96, steps=300),
                "debye_slabs_192x192x96_pml10_6slabs_dft64x64x64")
    if name == "c1":
        return cases.pec_box(), "pec_box_40^3"
    raise ValueError(name)


def cell_counts(t):
    n = t["nx"] * t["ny"] * t["nz"]
    npml = int(t["n_pml_cells"])
    mats = np.asarray(t["sp_material"])
    nmat = int((mats > 0).sum())
    orders = np.zeros(max(int(t["n_materials"]), 1), dtype=np.int64)
    if int(t["n_materials"]):
        orders = (np.asarray(t["mat_eps_order"]) * np.asarray(t["mat_eps_exists"]) +
                  np.asarray(t["mat_mu_order"]) * np.asarray(t["mat_mu_exists"]))
    filt_taps = int(sum(orders[m - 1] for m in mats[mats > 0])) if nmat else 0
    return n, npml, nmat, filt_taps


def algorithmic_bytes(t, esz):
    """Bytes per step that the fused single-pass algorithm must move:
    12 link reads + 12 link writes per cell, +18 PML state values read and
    written per PML cell, +3 filter taps (FP64) read and written per filter
    order per dispersive cell, +16 B per DFT accumulator."""
    n, npml, nmat, taps = cell_counts(t)
    links = n * 24 * esz
    pml = npml * 36 * esz
    filt = taps * 3 * 16
    dft = int(t["dft_face_ptr"][-1]) * 16 if int(t["n_dft"]) else 0
    return dict(total=links + pml + filt + dft, bulk=(n - npml - nmat) * 24 * esz,
                special=(npml + nmat) * 24 * esz + pml + filt)


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def dist_setup(backend: str = ""):
    """One process per GPU (torchrun env).  NCCL on GPUs; gloo when no GPU is
    visible (the host-side replica logic is tested that way)."""
    world, rank, local = dist_env()
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        if not backend:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    v = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(v, op=dist.ReduceOp.MAX)
    return float(v.item())


def replica_rate(cells: int, steps: int, world: int, local_ms: float) -> tuple:
    """Whole-job rate of ``world`` replicas that each advance ``cells`` for
    ``steps``: total cell updates / the slowest rank's time.  Returns
    (Gcell-updates/s, max ms)."""
    ms = max_over_ranks(local_ms, world)
    return cells * steps * world / (ms / 1e3) / 1e9, ms


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_oracle_rate(t, budget_s: float, max_steps: int, threads: int = 1):
    """Time the CPU oracle (the C restatement of the reference's loop, its
    z-planes shared among ``threads`` host threads as the reference's MPI
    build shares z-slabs among ranks) on the same tables for a bounded number
    of steps; returns (Gcell/s, steps, s, threads used)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    o = oracle.Oracle(t, threads=threads)
    n = t["nx"] * t["ny"] * t["nz"]
    o.run(1)  # warm-up step (page-in)
    steps, t0 = 0, time.perf_counter()
    while steps < max_steps:
        o.run(1)
        steps += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    used = o.threads
    o.close()
    return n * steps / el / 1e9, steps, el, used


def workload_config(t, wname, world):
    n, npml, nmat, _ = cell_counts(t)
    return {"workload": wname, "cells": n, "pml_cells": npml, "material_cells": nmat,
            "n_timesteps": int(t["n_timesteps"]), "parallelism": f"replicas{world}",
            "l2": "inputs larger than L2 (126 MB): no flush"}


def run_reference_arm(args, world, rank):
    """The reference's CPU implementation of the path on this box's host
    cores.  The reference is Fortran and no Fortran compiler exists here, so
    the oracle (the plain-C restatement of its sequential loop, pinned by the
    reference's golden vectors) stands in for it, with all host threads."""
    if rank != 0:
        return
    from ggi_tlm_b200.problem import build_tables

    spec, wname = workload_spec(args.workload)
    t = build_tables(spec)
    budget = float(os.environ.get("TLM_REFERENCE_BUDGET_S", "60"))
    W = max(args.warmup, 3)
    rate, steps, el, used = cpu_oracle_rate(t, budget, max(args.steps, 1), host_threads())
    sample = (f"{steps} FP64 time steps of the full {t['nx']}x{t['ny']}x{t['nz']} mesh ({el:.1f} s) after 1 "
              f"untimed step")
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": world, "steps": steps,
        "warmup": W, "ms_per_step": el / steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(t, wname, world),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": used, "kind": "port", "sample": sample,
                         "note": "reference Fortran builds (SEQ, MPI) unavailable on this box (no Fortran "
                                 "compiler); the oracle's C restatement of the sequential loop, z-planes shared "
                                 "among host threads (the MPI build's z-slab split)"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def timed_solo(t, precision, device, K, W, world, finish=True, sample_clocks=False):
    """Advance one mesh: autotune on real steps, W warm-up steps, K timed
    steps (CUDA events on the launch stream, barriers around), then the rest
    of the solve untimed for the probe accuracy."""
    from ggi_tlm_b200 import autotune, capi
    from ggi_tlm_b200.problem import probe_series

    g = capi.GpuMesh(t, precision=precision, device=device)
    tv = autotune.tune(g, steps_per_variant=2, use_cache=False)
    g.run(W)
    g.set_timing(True)
    barrier(world)
    g.synchronize()
    sampler = ClockSampler(device) if sample_clocks else None
    if sampler:
        sampler.start()
    g.run(K)
    g.synchronize()
    clocks = sampler.stop() if sampler else None
    barrier(world)
    total, bulk = g.last_run_time()
    launches = g.last_run_launches()
    g.set_timing(False)
    probes = None
    if finish:
        g.run(t["n_timesteps"] - g.step)
        probes = probe_series(t, g.cell_output())
    mem = g.memory_bytes()
    g.close()
    return {"total_ms": total, "bulk_ms": bulk, "launches": launches, "clocks": clocks, "probes": probes,
            "variant": tv["variant"], "device_bytes": mem}


def probe_error(a, b):
    """Largest relative L2 error over the probes the wave has reached: a
    probe whose FP64 series stays below 1e-6 of the largest probe's holds
    only round-off (a short run), and its relative error means nothing."""
    norms = [float(np.linalg.norm(x)) for x in b]
    floor = 1e-6 * max(norms, default=0.0)
    errs = [float(np.linalg.norm(a[i] - b[i]) / norms[i]) for i in range(len(b)) if norms[i] > floor and norms[i] > 0]
    return max(errs) if errs else None


def bench_pair(t, device, peak, K=60, W=3):
    """FP32 and FP64 step rates of one mesh with the FP32 probe error over
    the complete solve (compact record for the section keys)."""
    from ggi_tlm_b200 import capi

    n = t["nx"] * t["ny"] * t["nz"]
    r32 = timed_solo(t, capi.TLM_PRECISION_FP32, device, K, W, 1)
    r64 = timed_solo(t, capi.TLM_PRECISION_FP64, device, K, W, 1)
    out = {}
    for key, r, esz in (("fp32", r32, 4), ("fp64", r64, 8)):
        ab = algorithmic_bytes(t, esz)
        out[key] = {"gcell_s": round(n * K / (r["total_ms"] / 1e3) / 1e9, 3),
                    "step_frac": round(ab["total"] / (r["total_ms"] / K / 1e3) / 1e9 / peak, 4),
                    "bulk_frac": round(ab["bulk"] / (r["bulk_ms"] / K / 1e3) / 1e9 / peak, 4)}
    out["fp32_probe_err"] = probe_error(r32["probes"], r64["probes"])
    out["steps"] = int(t["n_timesteps"])
    return out


def build_many(specs):
    """Tables of many problems, built in a pool of host processes (spawned,
    so no process inherits a CUDA context); table building is host work
    outside every timed region."""
    import multiprocessing as mp

    from ggi_tlm_b200.problem import build_tables

    n = max(1, min(len(specs), host_threads(), 32))
    if n == 1:
        return [build_tables(s) for s in specs]
    with mp.get_context("spawn").Pool(n) as pool:
        return pool.map(build_tables, specs, chunksize=1)


def bench_batch(device):
    """Config 4: 96 uneven PML boxes (edges U[24,160], 0-8 spheres, point
    sources, 1500-5000 steps) advanced together, FP32, against the same boxes
    solved one after another."""
    from ggi_tlm_b200 import capi, cases

    tabs = build_many(cases.batch_boxes())
    meshes = [capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP32, device=device) for t in tabs]
    b = capi.GpuBatch(meshes)
    # tune the batch kernel configuration on the first real steps
    tune = {}
    for v in (1, 3, 4):
        b.set_variant(v)
        b.run(8)
        ms, cu, _ = b.last_run()
        tune[v] = ms / 8
    best = min(tune, key=tune.get)
    b.set_variant(best)
    b.run(100000)
    ms, cu, launches = b.last_run()
    b.close()
    for g in meshes:
        g.close()
    # the same boxes one at a time (graph-replayed solo runs)
    solo_ms, solo_cu = 0.0, 0
    for t in tabs:
        with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP32, device=device) as g:
            g.set_variant(best)
            g.run(t["n_timesteps"])
            total, _ = g.last_run_time()
            solo_ms += total
            solo_cu += t["nx"] * t["ny"] * t["nz"] * t["n_timesteps"]
    steps = max(t["n_timesteps"] for t in tabs)
    return {"gcell_s": round(cu / (ms / 1e3) / 1e9, 3), "solo_gcell_s": round(solo_cu / (solo_ms / 1e3) / 1e9, 3),
            "speedup_vs_solo": round((cu / ms) / (solo_cu / solo_ms), 3) if solo_ms else None,
            "launches": launches, "launches_per_step": round(launches / max(steps - 24, 1), 2),
            "boxes": len(tabs), "variant": best,
            "note": "96 PML boxes, edges U[24,160], 0-8 spheres, 1500-5000 steps, FP32; the first 24 steps of "
                    "every box ran during variant tuning (same numerics)"}


def bench_serving(device, n_requests=256):
    """Config 5: Poisson arrivals (40/s, seeded) of solves with edges
    log-U[32,256], 0-3 Debye slabs, 6-10 cell PML, 1000-8000 steps, served
    by continuous batching under a 150 GB budget, against sequential
    plain-FP64 solves of the same trace.  Two policies: every request in
    FP32 (``fp32_all``), and a per-request precision chosen a priori by the
    fitted FP32 error bound against the 1e-4 tolerance (the headline keys:
    FP32 where the bound allows it, FP64 elsewhere, in one server)."""
    from ggi_tlm_b200 import capi, cases, serving

    tabs = build_many(cases.serving_requests(n_requests))
    trace = serving.poisson_trace(list(range(len(tabs))), rate_per_s=40.0, seed=7, build=lambda i: tabs[i])
    base_res = serving.sequential_fp64(trace, device=device)
    base = serving.summarize(base_res)

    def serve(choose):
        eng = serving.GpuEngine(device=device, variant=1, choose=choose)
        srv = serving.Server(engine=eng, budget_bytes=150e9, max_slots=64, quantum=64)
        res = srv.serve(trace)
        srv.engine.close()
        errs = [probe_error(a.probes, b_.probes) for a, b_ in zip(res, base_res)]
        errs = [e for e in errs if e is not None]
        return srv, serving.summarize(res), errs

    tol = 1e-4
    choose = serving.precision_by_error(serving.FP32_ERROR_MODEL, tol)
    n32 = sum(choose(t) == capi.TLM_PRECISION_FP32 for t in tabs)
    srv, ours, errs = serve(choose)
    _, all32, errs32 = serve(lambda t: capi.TLM_PRECISION_FP32)
    return {"ratio": round(ours["solves_per_s"] / base["solves_per_s"], 3),
            "solves_s": round(ours["solves_per_s"], 3), "fp64_seq_solves_s": round(base["solves_per_s"], 3),
            "p50_s": round(ours["latency_p50_s"], 3), "p95_s": round(ours["latency_p95_s"], 3),
            "p99_s": round(ours["latency_p99_s"], 3),
            "fp64_seq_p50_s": round(base["latency_p50_s"], 3), "fp64_seq_p99_s": round(base["latency_p99_s"], 3),
            "probe_err_max": max(errs) if errs else None, "tol": tol, "fp32_requests": int(n32),
            "solves": len(errs), "peak_slots": srv.peak_slots, "peak_gb": round(srv.peak_bytes / 1e9, 2),
            "fp32_all": {"ratio": round(all32["solves_per_s"] / base["solves_per_s"], 3),
                         "solves_s": round(all32["solves_per_s"], 3), "p50_s": round(all32["latency_p50_s"], 3),
                         "p99_s": round(all32["latency_p99_s"], 3),
                         "probe_err_max": max(errs32) if errs32 else None,
                         "probe_err_median": float(np.median(errs32)) if errs32 else None,
                         "over_tol": int(sum(e > tol for e in errs32))},
            "detail": {"routed": ours, "fp32_all": all32, "fp64_sequential": base,
                       "request_errors_fp32_all": [round(e, 9) for e in errs32]}}


def run_batch_workload(args):
    """``--workload c4``: the batched workload's step rate alone (the 96
    boxes advanced together for W + K steps, FP32 and FP64), one JSON line;
    small enough to run under a profiler's launch list."""
    from ggi_tlm_b200 import build, capi, cases

    build.build()
    tabs = build_many(cases.batch_boxes())
    cells = sum(t["nx"] * t["ny"] * t["nz"] for t in tabs)
    out = {"workload": "batch_boxes_96", "cells": int(cells), "steps": args.steps, "warmup": max(args.warmup, 3)}
    for key, prec in (("fp32", capi.TLM_PRECISION_FP32), ("fp64", capi.TLM_PRECISION_FP64)):
        meshes = [capi.GpuMesh(t, precision=prec) for t in tabs]
        b = capi.GpuBatch(meshes)
        b.set_variant(int(os.environ.get("TLM_VARIANT", "1")))
        b.run(max(args.warmup, 3))
        b.run(args.steps)
        ms, cu, launches = b.last_run()
        out[key] = {"gcell_s": round(cu / (ms / 1e3) / 1e9, 3), "ms_per_step": round(ms / args.steps, 4),
                    "launches_per_step": launches / args.steps}
        b.close()
        for g in meshes:
            g.close()
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="t512", choices=["t512", "t192", "c2", "c3", "c3h", "c1", "c4"],
                    help="c4: the batched workload's step rate alone (one JSON line of its own)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--quick", action="store_true", help="main workload only (no C2, C3, batch, serving sections)")
    ap.add_argument("--serving-requests", type=int, default=256)
    args = ap.parse_args()
    if args.impl == "reference":  # rank 0 alone; no process group, no collective
        world, rank, _ = dist_env()
        run_reference_arm(args, world, rank)
        return
    if args.workload == "c4":
        run_batch_workload(args)
        return
    world, rank, local = dist_setup()

    from ggi_tlm_b200 import build, capi
    from ggi_tlm_b200.problem import build_tables

    build.build()
    spec, wname = workload_spec(args.workload)
    t = build_tables(spec)
    K, W = args.steps, max(args.warmup, 3)
    if K + W + 40 > t["n_timesteps"]:
        K = t["n_timesteps"] - W - 40
    n = t["nx"] * t["ny"] * t["nz"]
    peak, peak_kind = measured_peak()

    # headline: the plain FP64 path (the reference's precision); then the FP32 fast path
    r64 = timed_solo(t, capi.TLM_PRECISION_FP64, local, K, W, world, sample_clocks=True)
    value, ms_max = replica_rate(n, K, world, r64["total_ms"])
    r32 = timed_solo(t, capi.TLM_PRECISION_FP32, local, K, W, world)
    v32, ms32 = replica_rate(n, K, world, r32["total_ms"])
    ab64, ab32 = algorithmic_bytes(t, 8), algorithmic_bytes(t, 4)
    bulk_gbs = ab64["bulk"] / (r64["bulk_ms"] / K / 1e3) / 1e9
    step64 = ab64["total"] / (r64["total_ms"] / K / 1e3) / 1e9
    step32 = ab32["total"] / (r32["total_ms"] / K / 1e3) / 1e9
    bulk32 = ab32["bulk"] / (r32["bulk_ms"] / K / 1e3) / 1e9
    err32 = probe_error(r32["probes"], r64["probes"])

    # end to end through the C-ABI with host buffers, FP64: create + table
    # upload, every step tlm_gpu_run(t, 1) + read-back of that step's probe
    # samples, DFT read-back at the end
    e2e = None
    if not args.no_e2e:
        barrier(world)
        t0 = time.perf_counter()
        NE = int(t["n_timesteps"])
        g = capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP64, device=local)
        row = np.zeros((1, max(int(t["n_out_cells"]), 1), 6))
        for s_ in range(NE):
            g.run(1, sync=False)
            capi._check(capi._lib.tlm_gpu_fetch_cell_output(g.h, s_ + 1, 1, row.ctypes.data_as(capi._f64p)))
        dft = g.dft()
        g.close()
        e2e_s = max_over_ranks(time.perf_counter() - t0, world)
        table_bytes = sum(np.asarray(v).nbytes for k, v in t.items() if isinstance(v, np.ndarray))
        e2e = {"value": n * NE * world / e2e_s / 1e9, "unit": UNIT, "steps": NE,
               "h2d_bytes_per_step": int(table_bytes / NE),
               "d2h_bytes_per_step": int(int(t["n_out_cells"]) * 6 * 8 + dft.nbytes / NE),
               "dtype": "f64",
               "includes": "a whole FP64 solve through the C-ABI from host buffers: handle create, table upload, "
                           "every step tlm_gpu_run + read-back of that step's probe samples, DFT read-back"}

    sections = not args.quick and world == 1  # per-GPU sections, reported at N=1
    c2 = c3 = c4 = c5 = None
    if sections:
        c2 = bench_pair(build_tables(workload_spec("c2")[0]), local, peak)
        c3 = bench_pair(build_tables(workload_spec("c3")[0]), local, peak)
        c4 = bench_batch(local)
        c5 = bench_serving(local, args.serving_requests)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, steps, el, used = cpu_oracle_rate(t, float(os.environ.get("TLM_CPU_BUDGET_S", "20")), 1000,
                                                host_threads())
        cpu = {"value": rate, "unit": UNIT, "cores": used, "kind": "port",
               "sample": f"{steps} FP64 time steps of the same {t['nx']}x{t['ny']}x{t['nz']} mesh ({el:.1f} s), "
                         f"oracle z-planes shared among {used} host threads"}

    if rank == 0:
        nm = NCU_TRAFFIC.get(wname, {})
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "fp32": {"value": v32, "ms_per_step": ms32 / K, "step_frac": step32 / peak, "bulk_frac": bulk32 / peak,
                     "step_frac_of_8tbs": step32 / 8000.0, "probe_rel_l2_vs_fp64_max": err32,
                     "probe_steps": int(t["n_timesteps"]), "variant": r32["variant"]},
            "fp64_step_frac": step64 / peak,
            "c2": c2, "c3": c3,
            "c4": {k: v for k, v in c4.items() if k != "note"} if c4 else None,
            "c5": {k: v for k, v in c5.items() if k != "detail"} if c5 else None,
            "config": dict(workload_config(t, wname, world),
                           precision="fp64 everywhere (headline); fp32 links with fp64 filters, PML recursion and "
                                     "DFT (fp32 key)",
                           bulk_variant_fp64=r64["variant"], bulk_variant_fp32=r32["variant"]),
            "roofline": {"bound": "hbm", "kernel": bulk_kernel_name(r64["variant"], 2),
                         "achieved": bulk_gbs, "peak": peak, "unit": "GB/s", "frac": bulk_gbs / peak,
                         "peak_kind": peak_kind,
                         "traffic": (nm["bytes_per_cell"] * ab64["bulk"] / 192) if nm.get("bytes_per_cell") else None,
                         "traffic_source": nm.get("source"),
                         "algorithmic_bytes_per_launch": ab64["bulk"], "avg_launch_ms": r64["bulk_ms"] / K},
            "step_roofline": {"achieved": step64, "frac": step64 / peak,
                              "algorithmic_bytes_per_step": ab64["total"], "frac_of_8tbs": step64 / 8000.0},
            "e2e": e2e, "cpu_baseline": cpu, "gpu_launches": r64["launches"], "clocks": r64["clocks"],
            "device_bytes": r64["device_bytes"],
            "c4_note": c4.get("note") if c4 else None,
            "c5_detail": c5.get("detail") if c5 else None,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
