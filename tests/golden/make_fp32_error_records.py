"""Measure the FP32 path's probe error on a serving trace (needs a GPU) and
store it as the fixture the FP32 error model is fitted on
(tests/golden/fp32_error_records_seed<S>.json).

Each request of ``cases.serving_requests(n, seed=S)`` is solved alone in
FP32 and in FP64 through the library; per centre output point the record
holds ``serving.fp32_error_features`` and the relative L2 error of the FP32
series against the FP64 one over the complete solve.  The seed differs from
the one the serving benchmark's trace uses, so the model that routes the
benchmark's requests was not fitted on them.

    python tests/golden/make_fp32_error_records.py [n_requests] [seed]
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from ggi_tlm_b200 import build, capi, cases, serving  # noqa: E402
from ggi_tlm_b200.problem import build_tables, probe_series  # noqa: E402


def main():
    n = int(sys.argv[1]) if len(sys.argv) > 1 else 256
    seed = int(sys.argv[2]) if len(sys.argv) > 2 else 8
    build.build()
    capi.load_library()
    records = []
    for i, spec in enumerate(cases.serving_requests(n, seed=seed)):
        t = build_tables(spec)
        series = {}
        for prec in (capi.TLM_PRECISION_FP32, capi.TLM_PRECISION_FP64):
            with capi.GpuMesh(t, precision=prec) as g:
                g.run(int(t["n_timesteps"]))
                series[prec] = probe_series(t, g.cell_output())
        a, b = series[capi.TLM_PRECISION_FP32], series[capi.TLM_PRECISION_FP64]
        errs = [float(np.linalg.norm(a[k] - b[k]) / np.linalg.norm(b[k])) if np.linalg.norm(b[k]) > 0 else 0.0
                for k in range(len(b))]
        records.append({"request": i, "features": serving.fp32_error_features(t).round(6).tolist(),
                        "errors": [float("%.4e" % e) for e in errs]})
        print(i, max(errs) if errs else None, flush=True)
    out = os.path.join(HERE, f"fp32_error_records_seed{seed}.json")
    with open(out, "w") as f:
        json.dump({"seed": seed, "n_requests": n, "records": records}, f, separators=(",", ":"))
    print("wrote", out)


if __name__ == "__main__":
    main()
