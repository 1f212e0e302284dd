"""The served form on the GPU: jobs of different sizes, durations and
plasticity, arriving while others run, give each the raster (SHA-256 of its
spikes, step by step) and the synaptic event count it gives alone."""
import importlib

import pytest

from tests.conftest import package

pytestmark = pytest.mark.gpu
S = importlib.import_module(package().__name__ + ".serve")
nc = importlib.import_module(package().__name__ + ".netconfig")


def jobs():
    specs = [  # side, ms, arrival s, seed, stdp
        (1, 180, 0.0, 3, False), (2, 120, 0.0, 4, True), (3, 90, 0.05, 5, False),
        (1, 60, 0.1, 6, True), (2, 150, 0.2, 7, False), (4, 70, 0.2, 8, False),
    ]
    out = []
    for i, (side, ms, arr, seed, stdp) in enumerate(specs):
        cfg = nc.cortical_grid(side, side, total_ms=ms + 1, seed=seed, glob_h=side * side, stdp=stdp,
                               start_plasticity_ms=0, **({"p1": 0.0376} if side == 2 else {}))
        out.append(S.Job(job_id=i, cfg=cfg, duration_ms=ms, arrival_s=arr))
    return out


def test_each_result_is_the_same_alone_and_in_the_mix():
    served = S.Server(device=0, hbm_budget=150e9, max_slots=4, round_ms=16).run(jobs())
    alone = S.run_one_at_a_time(jobs(), device=0, read_ms=40)
    for a, b in zip(served, alone):
        assert not a.error and not b.error
        assert a.steps_done == b.steps_done == a.duration_ms
        assert a.raster_sha256 == b.raster_sha256 and a.spikes == b.spikes and a.events == b.events
        assert a.latency_s >= a.real_time_factor * a.duration_ms * 1e-3 > 0
    # more jobs than slots: some waited for a slot, and ran while others ran
    starts = sorted(j.t_start for j in served)
    dones = sorted(j.t_done for j in served)
    assert starts[-1] >= dones[0]
    assert any(x.t_start < y.t_done and y.t_start < x.t_done for x in served for y in served if x is not y)
