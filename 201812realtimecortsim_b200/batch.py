"""The batched form: many independent networks of uneven size (a parameter
sweep over seeds, external rate and adaptation strength) stepped together.

* build      -- the networks are built from several host threads at once
                (each build is stream-ordered on its own engine: builds
                overlap on the device);
* graph      -- 80 steps of every network, queued one step of each network
                at a time (dpsnn_step_many's order), are recorded once into a
                CUDA graph (dpsnn_graph_create); a run of the graph is one
                launch that advances every network by 80 steps;
* autotune   -- the delivery, warp-sort and heavy-run kernels of a small
                network waste most of their default grids (sized for a whole
                GPU) on idle blocks; :func:`autotune` records the batch with
                each candidate grid rule, times graph runs, and keeps the
                fastest.  Grids change launch counts only: the results are
                the same (every kernel loops over its work).

Each network's raster is the one it gives alone (a GPU test checks this).
The reference has no batched form: a sweep is that many separate runs.
"""
from __future__ import annotations

import concurrent.futures
import time
from typing import Callable, List, Sequence

import numpy as np

from . import engine as E
from . import netconfig as nc

__all__ = ["sweep_configs", "build_all", "shape_rule", "autotune", "BatchRunner", "GRAPH_STEPS", "CANDIDATES"]

GRAPH_STEPS = 80   # steps per graph run (a multiple of the engine's 80-step spike ring)


def sweep_configs(n: int, total_ms: int, seed: int = 2024, sides=(1, 2, 3, 4)) -> List[nc.NetConfig]:
    """The batched sweep: grid side uniform over ``sides``; per network its
    own seed, external Poisson rate (1-5 kHz: NuExt 1-5 Hz over CExt 1000)
    and calcium adaptation increment (0-2x the baseline 1.0); one reference
    rank per cortical module; the delay-range sub-population, so that no
    network is refused for a delay level of 80."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        g = int(rng.choice(sides))
        nu, alpha = float(rng.uniform(1.0, 5.0)), float(rng.uniform(0.0, 2.0))
        kw = {"p1": 0.0376} if g == 2 else {}
        out.append(nc.cortical_grid(g, g, total_ms=total_ms, seed=1 + i, nu_ext_hz=nu, alpha_c=alpha,
                                    glob_h=g * g, delay_range_subpop=True, **kw))
    return out


def build_all(cfgs: Sequence[nc.NetConfig], device: int = 0, threads: int = 16) -> List[E.Engine]:
    """Engines for ``cfgs``, built from ``threads`` host threads at once."""
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(threads, len(cfgs)))) as pool:
        return list(pool.map(lambda c: E.Engine(c, device=device), cfgs))


def shape_rule(blocks_per_module: int) -> Callable[[E.Engine, nc.NetConfig], tuple]:
    """A grid rule: the three kernels' blocks in proportion to the network's
    modules (0 = the engine's defaults)."""
    def rule(eng, cfg):
        if blocks_per_module <= 0:
            return (0, 0, 0)
        b = max(4, blocks_per_module * cfg.n_modules)
        return (b, b, 2 * b)
    rule.blocks_per_module = blocks_per_module
    return rule


CANDIDATES = (4, 16, 64, 0)   # blocks per module; 0 = defaults


def _time_graph_runs(engines, runs: int, sync: Callable[[], None]) -> float:
    g = E.Graph(engines, GRAPH_STEPS)
    try:
        g.run()      # first run: warm
        sync()
        t0 = time.perf_counter()
        for _ in range(runs):
            g.run()
        sync()
        return (time.perf_counter() - t0) / runs
    finally:
        g.close()


def autotune(engines: Sequence[E.Engine], cfgs: Sequence[nc.NetConfig], sync: Callable[[], None],
             candidates=CANDIDATES, runs: int = 1) -> dict:
    """Pick the grid rule whose graph of the whole batch runs fastest.  Each
    candidate costs (1 + runs) graph runs of simulated steps; the engines
    keep the chosen shapes.  Returns {"blocks_per_module": best, "seconds":
    {candidate: seconds per graph run}, "steps": simulated steps used}."""
    times = {}
    for c in candidates:
        rule = shape_rule(c)
        for e, cfg in zip(engines, cfgs):
            e.set_launch_shape(*rule(e, cfg))
        times[c] = _time_graph_runs(engines, runs, sync)
    best = min(times, key=times.get)
    rule = shape_rule(best)
    for e, cfg in zip(engines, cfgs):
        e.set_launch_shape(*rule(e, cfg))
    return {"blocks_per_module": best, "seconds": times, "steps": len(candidates) * (1 + runs) * GRAPH_STEPS}


class BatchRunner:
    """Steps a batch of engines in graph runs of GRAPH_STEPS steps; the
    engines must have run their first step, at the same step count."""

    def __init__(self, engines: Sequence[E.Engine]):
        self.engines = list(engines)
        self.graph = E.Graph(self.engines, GRAPH_STEPS)

    def run(self, nsteps: int):
        if nsteps % GRAPH_STEPS:
            raise ValueError(f"the batch advances in runs of {GRAPH_STEPS} steps")
        for _ in range(nsteps // GRAPH_STEPS):
            self.graph.run()

    def close(self):
        self.graph.close()
