"""Serving loop: admission by HBM footprint, slots, continuous batching.

The scheduling logic is checked on the CPU with a stand-in engine; the GPU
test checks that every result is bit-identical alone and in the mix."""
import numpy as np
import pytest

from ggi_tlm_b200 import capi, cases, serving
from ggi_tlm_b200.problem import build_tables


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t


class FakeEngine:
    """Advances solves instantly; each quantum costs 0.01 s of fake time."""

    def __init__(self, clock):
        self.clock = clock
        self.steps = {}
        self.targets = {}
        self.max_concurrent = 0

    def add(self, rid, tables):
        self.steps[rid] = 0
        self.targets[rid] = tables["n_timesteps"]
        self.max_concurrent = max(self.max_concurrent, len(self.steps))

    def remove(self, rid):
        del self.steps[rid]

    def advance(self, n):
        for r in self.steps:
            self.steps[r] = min(self.targets[r], self.steps[r] + n)
        self.clock.t += 0.01

    def progress(self, rid):
        return self.steps[rid]

    def results(self, rid):
        return None, None


def small_tables(n, steps):
    return build_tables(cases.pml_point_source(n, steps=steps, pml=2, n_probes=1))


def test_admission_respects_budget_slots_and_order():
    clock = FakeClock()
    eng = FakeEngine(clock)
    tabs = [small_tables(10, 30 + 10 * i) for i in range(6)]
    fp = serving.footprint_bytes(tabs[0])
    trace = [serving.Request(i, 0.0, tabs[i]) for i in range(6)]
    srv = serving.Server(engine=eng, budget_bytes=2.5 * fp, max_slots=8, quantum=10, clock=clock)
    res = srv.serve(trace)
    assert [r.rid for r in res] == list(range(6))
    assert eng.max_concurrent == 2  # the budget admits two solves at a time
    assert srv.peak_bytes <= 2.5 * fp
    admits = [e[2] for e in srv.events if e[1] == "admit"]
    assert admits == sorted(admits)  # arrival order
    # a slot limit binds before the budget
    clock2 = FakeClock()
    eng2 = FakeEngine(clock2)
    srv2 = serving.Server(engine=eng2, budget_bytes=100 * fp, max_slots=3, quantum=10, clock=clock2)
    srv2.serve([serving.Request(i, 0.0, tabs[i]) for i in range(6)])
    assert eng2.max_concurrent == 3


def test_late_arrivals_join_running_batch():
    clock = FakeClock()
    eng = FakeEngine(clock)
    tabs = [small_tables(10, 200), small_tables(10, 50)]
    trace = [serving.Request(0, 0.0, tabs[0]), serving.Request(1, 0.05, tabs[1])]
    res = serving.Server(engine=eng, quantum=10, clock=clock).serve(trace)
    assert eng.max_concurrent == 2  # request 1 was admitted while request 0 was running
    assert res[1].finished < res[0].finished
    assert res[1].queue_wait < 0.011


def test_oversized_request_is_rejected():
    clock = FakeClock()
    t = small_tables(10, 10)
    with pytest.raises(ValueError):
        serving.Server(engine=FakeEngine(clock), budget_bytes=1000, clock=clock).serve([serving.Request(0, 0.0, t)])


@pytest.mark.gpu
def test_results_same_alone_and_in_the_mix(gpu_lib):
    specs = cases.serving_requests(n_requests=5, edge=(14, 30), steps=(60, 140), pml=(2, 3), seed=9)
    tabs = [build_tables(s) for s in specs]
    trace = [serving.Request(i, 0.002 * i, t) for i, t in enumerate(tabs)]
    srv = serving.Server(engine=serving.GpuEngine(variant=1), max_slots=3, quantum=16)
    mixed = srv.serve(trace)
    srv.engine.close()
    assert srv.peak_slots == 3
    for r, t in zip(mixed, tabs):
        with capi.GpuMesh(t, precision=capi.TLM_PRECISION_FP32) as g:
            g.set_variant(1)
            g.run(t["n_timesteps"])
            from ggi_tlm_b200.problem import probe_series
            alone = probe_series(t, g.cell_output())
            alone_dft = g.dft()
        assert np.array_equal(r.probes, alone)
        assert np.array_equal(r.dft, alone_dft)


def test_footprint_counts_optional_outputs():
    from ggi_tlm_b200.problem import Block, OutputSurface, OutputVolume

    base = cases.pml_point_source(20, steps=100, pml=3, n_probes=1)
    t0 = build_tables(base)
    base.output_surfaces = [OutputSurface("Ex", plane=(3, 10, (4, 16), (4, 16)))]
    base.output_volumes = [OutputVolume(Block(5, 14, 5, 14, 5, 14), "Ey", "field")]
    t1 = build_tables(base)
    extra = serving.footprint_bytes(t1) - serving.footprint_bytes(t0)
    # the two histories alone: 13*13 faces and 10^3 cells, 100 steps each, 8 bytes a value
    assert extra >= (13 * 13 + 1000) * 100 * 8


def test_fp32_error_features_geometry():
    """Features of a solve: steps, source distance, cells to the PML."""
    s = cases.pml_point_source(40, 30, 24, pml=4, steps=1000, n_probes=0)
    from ggi_tlm_b200.problem import OutputPoint
    s.outputs = [OutputPoint((20, 15, 12), "Ex"), OutputPoint((5, 15, 12), "Ex"), OutputPoint((3, 3, 3), "Ey")]
    t = build_tables(s)
    src = np.asarray(s.point_excitations[0].cell, dtype=float)
    f = serving.fp32_error_features(t)
    assert f.shape == (3, 3)
    np.testing.assert_allclose(f[:, 0], 3.0)
    np.testing.assert_allclose(10 ** f[0, 1], max(1.0, np.linalg.norm(src - (20, 15, 12))))
    # cells 1..4 are PML: cell 5 touches it (gap 0), cell 20 is 7 cells in along z (24 - 4 - 12 = 8, 12 - 5 = 7)
    np.testing.assert_allclose(10 ** f[:, 2] - 1, [7, 0, 0])


def test_fp32_error_fit_and_bound():
    """The fit recovers a planted power law; the bound adds the largest
    residual; the chooser routes by the bound."""
    rng = np.random.default_rng(1)
    coef = np.array([-7.0, 0.6, 0.8, -0.5])
    recs = []
    for _ in range(40):
        f = np.column_stack([rng.uniform(3, 3.9, 2), rng.uniform(0, 2, 2), rng.uniform(0, 1.5, 2)])
        e = 10 ** (coef[0] + f @ coef[1:] + rng.normal(0, 0.05, 2))
        recs.append({"features": f.tolist(), "errors": e.tolist()})
    m = serving.fit_fp32_error_model(recs)
    np.testing.assert_allclose(m["coef"], coef, atol=0.1)
    assert 0 < m["margin"] < 0.25 and m["n_points"] == 80
    t = small_tables(16, 1000)
    b = serving.fp32_error_bound(t, m)
    f = serving.fp32_error_features(t)
    assert b == pytest.approx(10 ** (np.max(m["coef"][0] + f @ np.asarray(m["coef"][1:])) + m["margin"]))
    assert serving.precision_by_error(m, tol=b * 1.01)(t) == capi.TLM_PRECISION_FP32
    assert serving.precision_by_error(m, tol=b * 0.99)(t) == capi.TLM_PRECISION_FP64
    longer = small_tables(16, 4000)
    assert serving.fp32_error_bound(longer, m) > b


def test_fp32_error_model_is_the_fit_of_the_measured_records():
    """The routing model is the fit of the FP32-vs-FP64 errors measured on a
    B200 over the 256 solves of a trace with another seed than the serving
    benchmark's (tests/golden/make_fp32_error_records.py)."""
    import json
    import os

    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fp32_error_records_seed8.json")
    d = json.load(open(path))
    assert d["seed"] == 8 and len(d["records"]) == 256
    m = serving.fit_fp32_error_model(d["records"])
    np.testing.assert_allclose(m["coef"], serving.FP32_ERROR_MODEL["coef"], rtol=1e-9)
    assert m["margin"] == pytest.approx(serving.FP32_ERROR_MODEL["margin"], rel=1e-9)
    # the features the records hold are the library's own, recomputed from the trace
    spec = cases.serving_requests(256, seed=8)[d["records"][3]["request"]]
    np.testing.assert_allclose(serving.fp32_error_features(build_tables(spec)), d["records"][3]["features"],
                               atol=1e-6)
