#!/usr/bin/env python
"""Benchmark of the B200 SCN-TLM time-stepping core.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload c2|t512|c3|c1]

One "step" is one TLM time step (excitation, scatter, connect, outer boundary,
face outputs, DFT) over the whole mesh.  Default workload: the 256^3
PML-bounded box with 32 dielectric spheres, a Huygens plane wave, 16 probes
and a 64-frequency 64x64-face FP64 DFT (seeded synthetic input), FP32 links.
The metric is cell-updates per second (whole job, all GPUs), with the fused
cell kernel's achieved HBM bandwidth against the measured copy peak.

Multi-GPU (torchrun, one process per GPU): the path does not shard here
(replicas only); every rank advances its own copy of the mesh, the timed
region is bracketed by barriers and the time is the max over ranks.
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

# DRAM bytes per launch of the bulk kernel (dram__bytes_read.sum +
# dram__bytes_write.sum) from one ncu --set full capture of the same workload.
NCU_TRAFFIC = {
    "pml_spheres_256^3_pml8_32spheres_huygens_dft64x64x64": {
        "bytes": 755.997440e6 + 609.044480e6,
        "source": "profiles/tlm_bulk_tma_kernel_pml_spheres_256_fp32.md (tlm_bulk_tma_kernel<float,4,512,3>)"},
    "debye_slabs_384x384x192_pml10_6slabs_dft64x64x64": {
        "bytes": None,
        "source": "no ncu capture of the bulk kernel on this workload; "
                  "profiles/tlm_special_kernel_debye_slabs_384x384x192_fp32.md covers its largest special kernel"},
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
    if name == "c3":
        return cases.debye_slabs(), "debye_slabs_384x384x192_pml10_6slabs_dft64x64x64"
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


def cpu_oracle_rate(t, budget_s: float, max_steps: int):
    """Time the CPU oracle (the C restatement of the reference's loop) on the
    same tables for a bounded number of steps; returns (Gcell/s, steps, s)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    o = oracle.Oracle(t)
    n = t["nx"] * t["ny"] * t["nz"]
    o.run(1)  # warm-up step (page-in)
    steps, t0 = 0, time.perf_counter()
    while steps < max_steps:
        o.run(1)
        steps += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    o.close()
    return n * steps / el / 1e9, steps, el


def run_reference_arm(args, world, rank):
    if rank != 0:
        return
    from ggi_tlm_b200.problem import build_tables

    spec, wname = workload_spec(args.workload)
    t = build_tables(spec)
    budget = float(os.environ.get("TLM_REFERENCE_BUDGET_S", "60"))
    rate, steps, el = cpu_oracle_rate(t, budget, max(args.steps, 1))
    sample = f"{steps} time steps of the full {t['nx']}x{t['ny']}x{t['nz']} mesh ({el:.1f} s)"
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": world, "steps": steps,
        "warmup": 1, "ms_per_step": el / steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wname, "cells": t["nx"] * t["ny"] * t["nz"]},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": 1, "kind": "port", "sample": sample,
                         "note": "reference Fortran build unavailable on this box (no Fortran compiler); "
                                 "single-threaded C restatement of its sequential loop"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _timed_steps(g, k):
    g.set_timing(True)
    g.run(k)
    total, bulk = g.last_run_time()
    g.set_timing(False)
    return total, bulk


def bench_target_512(device, peak):
    """The roofline target: 512^3 PML-bounded free-space mesh, point source."""
    from ggi_tlm_b200 import autotune, capi
    from ggi_tlm_b200.problem import build_tables, probe_series

    t = build_tables(__import__("ggi_tlm_b200.cases", fromlist=["x"]).pml_point_source(512, steps=2000))
    n = t["nx"] * t["ny"] * t["nz"]
    out = {"workload": "pml_point_source_512^3_pml8", "cells": n, "pml_cells": int(t["n_pml_cells"])}
    probes = {}
    for prec, esz, key in ((capi.TLM_PRECISION_FP32, 4, "fp32"), (capi.TLM_PRECISION_FP64, 8, "fp64")):
        g = capi.GpuMesh(t, precision=prec, device=device)
        tv = autotune.tune(g, steps_per_variant=2, use_cache=False)
        g.run(3)
        K = 60
        total, bulk = _timed_steps(g, K)
        g.run(t["n_timesteps"] - g.step)  # untimed: the rest of the solve, for the probe accuracy
        probes[key] = probe_series(t, g.cell_output())
        g.close()
        ab = algorithmic_bytes(t, esz)
        step_gbs = ab["total"] / (total / K / 1e3) / 1e9
        out[key] = {"gcell_per_s": n * K / (total / 1e3) / 1e9, "ms_per_step": total / K,
                    "step_achieved_gbs": step_gbs, "step_frac_of_measured_hbm": step_gbs / peak,
                    "step_frac_of_8tbs": step_gbs / 8000.0,
                    "bulk_kernel_gbs": ab["bulk"] / (bulk / K / 1e3) / 1e9,
                    "bulk_kernel_frac_of_measured_hbm": ab["bulk"] / (bulk / K / 1e3) / 1e9 / peak,
                    "variant": tv["variant"], "timed_steps": K}
    a, b = probes["fp32"], probes["fp64"]
    errs = [float(np.linalg.norm(a[i] - b[i]) / np.linalg.norm(b[i])) for i in range(len(b)) if np.linalg.norm(b[i]) > 0]
    out["probe_rel_l2_fp32_vs_fp64_max"] = max(errs)
    out["probe_rel_l2_fp32_vs_fp64_median"] = float(np.median(errs))
    out["probe_steps"] = int(t["n_timesteps"])
    return out


def bench_batch(device):
    """Config 4: 96 uneven PML boxes (edges U[24,160], 0-8 spheres, point
    sources, 1500-5000 steps) advanced together, FP32, against the same boxes
    solved one after another."""
    from ggi_tlm_b200 import capi, cases
    from ggi_tlm_b200.problem import build_tables

    specs = cases.batch_boxes()
    tabs = [build_tables(s) for s in specs]
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
    return {"workload": "96 PML boxes, edges U[24,160], 0-8 spheres, 1500-5000 steps, FP32",
            "boxes": len(tabs), "cell_updates": cu, "gcell_per_s": cu / (ms / 1e3) / 1e9, "device_ms": ms,
            "variant": best, "variant_ms_per_step": tune, "kernel_launches": launches,
            "solo_sequential_gcell_per_s": solo_cu / (solo_ms / 1e3) / 1e9,
            "speedup_vs_solo_sequential": (cu / ms) / (solo_cu / solo_ms) if solo_ms else None,
            "note": "first 24 steps of every box ran during variant tuning (same numerics)"}


def bench_serving(device, n_requests=32):
    """Config 5: Poisson arrivals (40/s, seeded) of solves with edges
    log-U[32,256], 0-3 Debye slabs, 6-10 cell PML, 1000-8000 steps; FP32
    continuous batching under a 150 GB budget against sequential plain-FP64
    solves of the same trace."""
    from ggi_tlm_b200 import cases, serving
    from ggi_tlm_b200.problem import build_tables

    specs = cases.serving_requests(n_requests)
    trace = serving.poisson_trace(specs, rate_per_s=40.0, seed=7, build=build_tables)
    srv = serving.Server(engine=serving.GpuEngine(device=device, variant=1), budget_bytes=150e9, max_slots=64,
                         quantum=64)
    res = srv.serve(trace)
    srv.engine.close()
    ours = serving.summarize(res)
    base_res = serving.sequential_fp64(trace, device=device)
    base = serving.summarize(base_res)
    errs = []
    for a, b_ in zip(res, base_res):
        for i in range(a.probes.shape[0]):
            nb = np.linalg.norm(b_.probes[i])
            if nb > 0:
                errs.append(float(np.linalg.norm(a.probes[i] - b_.probes[i]) / nb))
    return {"workload": f"{n_requests}-request Poisson trace, 40 req/s, edges log-U[32,256], 0-3 Debye slabs",
            "fp32_batched": ours, "fp64_sequential": base,
            "solves_per_s_ratio": ours["solves_per_s"] / base["solves_per_s"],
            "probe_rel_l2_vs_fp64_median": float(np.median(errs)) if errs else None,
            "probe_rel_l2_vs_fp64_max": float(np.max(errs)) if errs else None,
            "peak_slots": srv.peak_slots, "peak_bytes": srv.peak_bytes}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=["c2", "t512", "c3", "c1"])
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--quick", action="store_true", help="main workload only (no 512^3, batch, serving sections)")
    args = ap.parse_args()
    if args.impl == "reference":  # rank 0 alone; no process group, no collective
        world, rank, _ = dist_env()
        run_reference_arm(args, world, rank)
        return
    world, rank, local = dist_setup()

    from ggi_tlm_b200 import autotune, build, capi
    from ggi_tlm_b200.problem import build_tables, probe_series

    build.build()
    spec, wname = workload_spec(args.workload)
    t = build_tables(spec)
    K, W = args.steps, max(args.warmup, 3)
    if K + W + 40 > t["n_timesteps"]:
        K = t["n_timesteps"] - W - 40
    n, npml, nmat, taps = cell_counts(t)
    peak, peak_kind = measured_peak()

    tuned = {}

    def timed_run(precision, finish):
        g = capi.GpuMesh(t, precision=precision, device=local)
        tuned[precision] = autotune.tune(g, steps_per_variant=3, use_cache=False)  # real steps of the solve
        g.run(W)
        g.set_timing(True)
        barrier(world)
        g.synchronize()
        sampler = ClockSampler(local)
        sampler.start()
        g.run(K)
        g.synchronize()
        clocks = sampler.stop()
        barrier(world)
        total_ms, bulk_ms = g.last_run_time()
        launches = g.last_run_launches()
        probes = None
        if finish:  # untimed: complete the solve for the probe-accuracy comparison
            g.set_timing(False)
            g.run(t["n_timesteps"] - g.step)
            probes = probe_series(t, g.cell_output())
        mem = g.memory_bytes()
        g.close()
        return total_ms, bulk_ms, launches, clocks, probes, mem

    total32, bulk32, launches, clocks, p32, mem32 = timed_run(capi.TLM_PRECISION_FP32, not args.no_fp64)
    value, ms_max = replica_rate(n, K, world, total32)
    ab32 = algorithmic_bytes(t, 4)
    bulk_gbs = ab32["bulk"] / (bulk32 / K / 1e3) / 1e9
    step_gbs = ab32["total"] / (total32 / K / 1e3) / 1e9

    fp64 = None
    if not args.no_fp64:
        total64, bulk64, _, _, p64, mem64 = timed_run(capi.TLM_PRECISION_FP64, True)
        ab64 = algorithmic_bytes(t, 8)
        norms = [np.linalg.norm(p64[i]) for i in range(len(p64))]
        rel = max(np.linalg.norm(p32[i] - p64[i]) / norms[i] for i in range(len(p64)) if norms[i] > 0)
        fp64 = {"value": replica_rate(n, K, world, total64)[0], "unit": UNIT,
                "ms_per_step": total64 / K,
                "step_achieved_gbs": ab64["total"] / (total64 / K / 1e3) / 1e9,
                "step_frac_of_measured_hbm": ab64["total"] / (total64 / K / 1e3) / 1e9 / peak,
                "bulk_kernel_achieved_gbs": ab64["bulk"] / (bulk64 / K / 1e3) / 1e9,
                "probe_rel_l2_fp32_vs_fp64_max": rel, "probe_steps": int(t["n_timesteps"]),
                "device_bytes": mem64}

    # end to end through the C-ABI with host buffers: create + table upload,
    # every step tlm_gpu_run(t,1) + read back that step's probe samples, DFT read at the end
    barrier(world)
    t0 = time.perf_counter()
    NE = t["n_timesteps"] if not args.no_e2e else 0
    if NE:
        g = capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP32, device=local)
        row = np.zeros((1, max(int(t["n_out_cells"]), 1), 6))
        for s in range(NE):
            g.run(1, sync=False)
            capi._check(capi._lib.tlm_gpu_fetch_cell_output(g.h, s + 1, 1, row.ctypes.data_as(capi._f64p)))
        dft = g.dft()
        g.close()
        e2e_s = max_over_ranks(time.perf_counter() - t0, world)
        table_bytes = sum(np.asarray(v).nbytes for k, v in t.items() if isinstance(v, np.ndarray))
        e2e = {"value": n * NE * world / e2e_s / 1e9, "unit": UNIT, "steps": NE,
               "h2d_bytes_per_step": int(table_bytes / NE),
               "d2h_bytes_per_step": int(int(t["n_out_cells"]) * 6 * 8 + dft.nbytes / NE),
               "includes": "a whole solve through the C-ABI from host buffers: handle create, table upload, "
                           "every step tlm_gpu_run + read-back of that step's probe samples, DFT read-back"}
    else:
        e2e = None

    sections = not args.quick and world == 1  # per-GPU sections, reported at N=1
    t512 = bench_target_512(local, peak) if sections else None
    c4 = bench_batch(local) if sections else None
    c5 = bench_serving(local) if sections else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, steps, el = cpu_oracle_rate(t, float(os.environ.get("TLM_CPU_BUDGET_S", "20")), 1000)
        cpu = {"value": rate, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"{steps} time steps of the same {t['nx']}x{t['ny']}x{t['nz']} mesh ({el:.1f} s)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": wname, "cells": n, "pml_cells": npml, "material_cells": nmat,
                       "parallelism": f"replicas{world}", "precision": "fp32 links+scatter, fp64 filters+DFT",
                       "bulk_variant_fp32": tuned[capi.TLM_PRECISION_FP32]["variant"],
                       "bulk_variant_fp64": tuned.get(capi.TLM_PRECISION_FP64, {}).get("variant"),
                       "l2": "state (%.2f GB) larger than L2 (126 MB)" % (ab32["total"] / 1e9)},
            "roofline": {"bound": "hbm", "kernel": bulk_kernel_name(tuned[capi.TLM_PRECISION_FP32]["variant"], 4),
                         "achieved": bulk_gbs, "peak": peak,
                         "unit": "GB/s", "frac": bulk_gbs / peak, "peak_kind": peak_kind,
                         "traffic": NCU_TRAFFIC.get(wname, {}).get("bytes"),
                         "traffic_source": NCU_TRAFFIC.get(wname, {}).get("source"),
                         "algorithmic_bytes_per_launch": ab32["bulk"],
                         "avg_launch_ms": bulk32 / K},
            "step_roofline": {"achieved": step_gbs, "frac": step_gbs / peak,
                              "algorithmic_bytes_per_step": ab32["total"]},
            "fp64": fp64, "e2e": e2e, "cpu_baseline": cpu, "gpu_launches": launches, "clocks": clocks,
            "target_512": t512, "batch_c4": c4, "serving_c5": c5,
            "device_bytes": mem32,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
