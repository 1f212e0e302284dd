"""The served form's request loop on the CPU (no GPU): admission by memory
footprint and slots, first come first served, slot release on completion,
results independent of the mix -- with stand-in engines whose spikes are a
function of their own network and step."""
import threading

import numpy as np
import pytest

from tests.conftest import package
import importlib

S = importlib.import_module(package().__name__ + ".serve")
nc = importlib.import_module(package().__name__ + ".netconfig")


class FakeEngine:
    live = 0
    peak = 0
    lock = threading.Lock()

    def __init__(self, cfg, device):
        if cfg.seed < 0:
            raise RuntimeError("dpsnn_create failed (-5): refused")
        self.seed, self.n, self.t = cfg.seed, cfg.glob_n, 0
        self.device_bytes = 1000
        with FakeEngine.lock:
            FakeEngine.live += 1
            FakeEngine.peak = max(FakeEngine.peak, FakeEngine.live)

    def step(self, k):
        self.t += k

    def spikes_range(self, t0, n):
        assert t0 + n <= self.t
        ids, te, cnt = [], [], []
        for t in range(t0, t0 + n):
            k = (self.seed * 31 + t) % 4
            ids += [(self.seed + t + i) % self.n for i in range(k)]
            te += [t - 0.25 * (i + 1) for i in range(k)]
            cnt.append(k)
        return np.array(ids, np.uint32), np.array(te, np.float64), np.array(cnt, np.uint32)

    def events_delivered(self):
        return 10 * self.t

    def close(self):
        with FakeEngine.lock:
            FakeEngine.live -= 1


def fake_step_many(engines, n):
    for e in engines:
        e.step(n)


def jobs(specs):
    out = []
    for i, (side, dur, arr, seed) in enumerate(specs):
        cfg = nc.cortical_grid(side, side, total_ms=dur, seed=seed)
        out.append(S.Job(job_id=i, cfg=cfg, duration_ms=dur, arrival_s=arr))
    return out


def server(**kw):
    FakeEngine.live = FakeEngine.peak = 0
    return S.Server(engine_factory=FakeEngine, step_many=fake_step_many, **kw)


def test_results_are_those_of_each_job_alone():
    specs = [(1, 130, 0.0, 3), (2, 77, 0.0, 4), (1, 200, 0.01, 5), (3, 45, 0.02, 6)]
    mixed = server(round_ms=16).run(jobs(specs))
    for j in mixed:
        alone = server(round_ms=64, max_slots=1).run(jobs([specs[j.job_id]]))[0]
        assert j.raster_sha256 == alone.raster_sha256 and j.spikes == alone.spikes
        assert j.events == 10 * j.duration_ms and j.steps_done == j.duration_ms
        assert j.t_done >= j.t_start >= j.t_admit >= j.arrival_s - 1e-9


def test_memory_budget_bounds_the_resident_jobs():
    js = jobs([(1, 60, 0.0, k + 1) for k in range(6)])
    for j in js:
        j.footprint = 100
    srv = server(hbm_budget=250, round_ms=8)
    srv.run(js)
    assert FakeEngine.peak == 2 and all(j.t_done is not None and not j.error for j in js)


def test_slots_bound_the_resident_jobs_and_free_on_completion():
    js = jobs([(1, 30 + 10 * k, 0.0, k + 1) for k in range(5)])
    srv = server(max_slots=3, round_ms=10)
    srv.run(js)
    assert FakeEngine.peak == 3
    # the two jobs admitted last could start only when earlier ones finished
    firsts = sorted(js, key=lambda j: j.t_admit)[:3]
    lasts = sorted(js, key=lambda j: j.t_admit)[3:]
    assert min(j.t_admit for j in lasts) >= min(j.t_done for j in firsts)


def test_first_come_first_served():
    # a large job at the head of the queue is not overtaken by a small one
    js = jobs([(1, 100, 0.0, 1), (2, 50, 0.001, 2), (1, 20, 0.002, 3)])
    js[0].footprint, js[1].footprint, js[2].footprint = 60, 60, 10
    import time
    while time.monotonic() < 0:   # arrivals are relative to the run's start
        pass
    server(hbm_budget=100, round_ms=10).run(js)
    assert js[2].t_admit >= js[1].t_admit


def test_oversized_and_refused_jobs_are_reported():
    js = jobs([(1, 20, 0.0, 1), (1, 20, 0.0, -1), (1, 20, 0.0, 2)])
    js[0].footprint = 10 ** 15
    out = server(hbm_budget=10 ** 9).run(js)
    assert "exceeds the budget" in out[0].error and out[0].t_done is None
    assert "refused" in out[1].error
    assert not out[2].error and out[2].steps_done == 20


def test_round_length_is_bounded_by_the_spike_ring():
    with pytest.raises(ValueError):
        S.Server(round_ms=100)


def test_request_stream_shape():
    js = S.poisson_jobs(200, rate_per_s=50.0, seed=3)
    arr = np.array([j.arrival_s for j in js])
    assert np.all(np.diff(arr) > 0) and 2.5 < arr[-1] < 6.0          # ~4 s of arrivals at 50/s
    sides = np.array([j.cfg.cfx for j in js])
    assert sides.min() >= 1 and sides.max() <= 16 and (sides == 1).sum() > (sides == 16).sum()
    durs = np.array([j.duration_ms for j in js])
    assert durs.min() >= 500 and durs.max() <= 10000
    assert 0.1 < np.mean([j.cfg.stdp is not None for j in js]) < 0.3


def test_footprint_estimate_grows_with_the_network():
    a = S.estimate_device_bytes(nc.cortical_grid(2, 2))
    b = S.estimate_device_bytes(nc.cortical_grid(4, 4, delay_range_subpop=True))
    c = S.estimate_device_bytes(nc.cortical_grid(4, 4, delay_range_subpop=True, stdp=True))
    assert 0 < a < b < c
    # ~5.6 M synapses at 2x2 (mean in-degree ~1125)
    assert 5.0e6 < S.expected_synapses(nc.cortical_grid(2, 2)) < 6.2e6
