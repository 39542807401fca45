"""Project autotuner for the bulk cell kernel.

The search space is the set of kernel configurations the library exposes
(``tlm_gpu_num_variants``): the register-pipelined kernel and TMA-staged
persistent kernels with different tile sizes (cells per block) and
shared-memory ring depths (plane staging depth).  All configurations give
bit-identical results, so the tuner runs on the live solve: it advances the
real mesh a few steps with each configuration, times them with CUDA events
on the launch stream, and keeps the fastest.  No step is wasted.

Choices are cached in a JSON file (``TLM_AUTOTUNE_CACHE``, default
``ggi_tlm_b200/_lib/autotune.json``) keyed by precision and mesh shape.
"""
from __future__ import annotations

import json
import os
from typing import Dict, Optional

from . import capi

_DEFAULT_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "autotune.json")


def _cache_path() -> str:
    return os.environ.get("TLM_AUTOTUNE_CACHE", _DEFAULT_CACHE)


def _key(mesh: "capi.GpuMesh") -> str:
    t = mesh.t
    n = t["nx"] * t["ny"] * t["nz"]
    frac = int(round(10 * (int(t["n_special"]) / max(n, 1))))
    return f"p{mesh.precision}_{t['nx']}x{t['ny']}x{t['nz']}_s{frac}"


def load_cache() -> Dict[str, dict]:
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except Exception:
        return {}


def save_cache(c: Dict[str, dict]):
    p = _cache_path()
    try:
        os.makedirs(os.path.dirname(p), exist_ok=True)
        tmp = p + ".tmp"
        with open(tmp, "w") as f:
            json.dump(c, f, indent=1, sort_keys=True)
        os.replace(tmp, p)
    except OSError:
        pass


def tune(mesh: "capi.GpuMesh", steps_per_variant: int = 2, use_cache: bool = True,
         max_steps: Optional[int] = None) -> dict:
    """Pick the fastest bulk-kernel configuration for ``mesh`` by running
    real steps of its solve.  Returns {"variant", "ms": {variant: ms/step},
    "steps_used", "cached"}."""
    forced = os.environ.get("TLM_VARIANT")
    if forced is not None:  # a fixed configuration (profiler runs, where trial timings mislead)
        mesh.set_variant(int(forced))
        return {"variant": int(forced), "ms": {}, "cached": False, "steps_used": 0}
    key = _key(mesh)
    cache = load_cache() if use_cache else {}
    if use_cache and key in cache:
        mesh.set_variant(int(cache[key]["variant"]))
        return dict(cache[key], cached=True, steps_used=0)
    remaining = mesh.t["n_timesteps"] - mesh.step
    if max_steps is not None:
        remaining = min(remaining, max_steps)
    nv = capi.num_variants()
    times = {}
    used = 0
    for v in range(nv):
        if used + steps_per_variant + 1 > remaining:
            break
        mesh.set_variant(v)
        mesh.run(1)  # configuration + first launch outside the timed steps
        mesh.set_timing(True)
        mesh.run(steps_per_variant)
        total, _ = mesh.last_run_time()
        mesh.set_timing(False)
        times[v] = total / steps_per_variant
        used += steps_per_variant + 1
    best = min(times, key=times.get) if times else 1
    mesh.set_variant(best)
    rec = {"variant": best, "ms": {str(k): v for k, v in times.items()}}
    if use_cache and times:
        cache = load_cache()
        cache[key] = rec
        save_cache(cache)
    return dict(rec, cached=False, steps_used=used)
