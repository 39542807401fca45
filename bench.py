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
    12 link reads + 12 link writes per cell, +24 PML state values read and
    written per PML cell, +3 filter taps (FP64) read and written per filter
    order per dispersive cell, +16 B per DFT accumulator."""
    n, npml, nmat, taps = cell_counts(t)
    links = n * 24 * esz
    pml = npml * 48 * esz
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


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
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

    v = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(v, op=dist.ReduceOp.MAX)
    return float(v.item())


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
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference_arm(args, world, rank)
        return

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
    ms_max = max_over_ranks(total32, world)
    value = n * K * world / (ms_max / 1e3) / 1e9
    ab32 = algorithmic_bytes(t, 4)
    bulk_gbs = ab32["bulk"] / (bulk32 / K / 1e3) / 1e9
    step_gbs = ab32["total"] / (total32 / K / 1e3) / 1e9

    fp64 = None
    if not args.no_fp64:
        total64, bulk64, _, _, p64, mem64 = timed_run(capi.TLM_PRECISION_FP64, True)
        ab64 = algorithmic_bytes(t, 8)
        norms = [np.linalg.norm(p64[i]) for i in range(len(p64))]
        rel = max(np.linalg.norm(p32[i] - p64[i]) / norms[i] for i in range(len(p64)) if norms[i] > 0)
        fp64 = {"value": n * K * world / (max_over_ranks(total64, world) / 1e3) / 1e9, "unit": UNIT,
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
            "roofline": {"bound": "hbm", "kernel": "tlm_cell_kernel<float,4>", "achieved": bulk_gbs, "peak": peak,
                         "unit": "GB/s", "frac": bulk_gbs / peak, "peak_kind": peak_kind,
                         "traffic": None,
                         "algorithmic_bytes_per_launch": ab32["bulk"],
                         "avg_launch_ms": bulk32 / K},
            "step_roofline": {"achieved": step_gbs, "frac": step_gbs / peak,
                              "algorithmic_bytes_per_step": ab32["total"]},
            "fp64": fp64, "e2e": e2e, "cpu_baseline": cpu, "gpu_launches": launches, "clocks": clocks,
            "device_bytes": mem32,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
