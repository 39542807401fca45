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
