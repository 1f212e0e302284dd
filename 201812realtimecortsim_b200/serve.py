"""The served form: simulation jobs of different sizes and durations taken as
they arrive, kept resident on the GPU, stepped together (continuous
batching).

The reference runs one network per set of MPI processes, blocking in its
``do fire() while`` loop until the run ends (DPSNN_mainUnderMPI.c:79-83).
Here one process serves a stream of such runs on one GPU:

* arrival    -- a job (a network description and a biological duration)
                joins the queue at its arrival time;
* admission  -- first come, first served: the job at the head of the queue is
                admitted when a slot is free and its device-memory footprint
                (estimated from the network's size, :func:`estimate_device_bytes`)
                fits under the budget beside the jobs already resident;
                later arrivals wait behind it;
* build      -- admitted jobs build their networks on worker threads (the
                build releases the interpreter lock), overlapping the
                stepping of the resident jobs;
* stepping   -- every round, all resident jobs advance together by
                ``round_ms`` steps through dpsnn_step_many (one step of every
                engine at a time, their kernels overlapping on the device);
                a job near its end takes its remaining steps only;
* results    -- each round's spike lists are read back per job (one wait per
                job and round, dpsnn_spikes_range) into the job's raster
                digest (SHA-256 of its spikes, step by step) and counts;
* completion -- a job that reached its duration is released at once: its
                slot and its device memory go to the next admissions.

A job's result depends only on its own network: engines share no state, so
the raster is the one the job gives alone (a GPU test checks this).
"""
from __future__ import annotations

import collections
import concurrent.futures
import dataclasses
import hashlib
import math
import time
from typing import Callable, List, Optional

import numpy as np

from . import engine as E
from . import netconfig as nc

__all__ = ["Job", "Server", "estimate_device_bytes", "expected_synapses", "poisson_jobs", "run_one_at_a_time"]


def expected_synapses(cfg: nc.NetConfig) -> float:
    """Expected synapse count of a network: every (source neuron, target
    sub-population, stencil cell inside the grid) contributes probability x
    target count (the generator's targets are independent draws)."""
    counts = [p.count for p in cfg.subpops]
    S = cfg.stencil_dim
    tot = 0.0
    for (s, t), (_, _, _, _, probs) in cfg.conn.items():
        if counts[s] == 0 or counts[t] == 0:
            continue
        acc = 0.0
        for cy in range(cfg.cfy):
            for cx in range(cfg.cfx):
                for dy in range(-(S - 1), S):
                    for dx in range(-(S - 1), S):
                        if 0 <= cx + dx < cfg.cfx and 0 <= cy + dy < cfg.cfy:
                            acc += probs[abs(dy) * S + abs(dx)]
        tot += acc * counts[s] * counts[t]
    return tot


def estimate_device_bytes(cfg: nc.NetConfig, events_per_neuron: int = 1024) -> int:
    """Device memory an engine of this network holds, from its size (the
    engine's layout: state, ring, event buckets, bath buffers, build scratch,
    6 B per synapse and 12 more with plasticity), with a 10 % margin on the
    synapse count."""
    N = cfg.glob_n
    cap = events_per_neuron
    while cap > 64 and 8 * cap * N > (16 << 30):
        cap //= 2
    max_ext = 0
    for p in cfg.subpops:
        if p.count and p.NuExt > 0:
            inv = 1000.0 / (p.NuExt * cfg.bath_cext)
            max_ext = max(max_ext, math.ceil(20 / inv))
    per_neuron = 66 + 2 * (cfg.D + 1) + 8 + 80 * 12 + 8 * cap + 20 + 12 + 2 * 9 * max_ext + 2 * 2 * cfg.D + 4
    per_syn = 6 + (12 if cfg.stdp is not None else 0)
    fixed = (116 << 20) + cfg.glob_h * 90_000 + cfg.n_modules * 2 * 7500 * 4
    return int(N * per_neuron + 1.1 * expected_synapses(cfg) * per_syn + fixed)


@dataclasses.dataclass
class Job:
    """One simulation request and, once served, its result and timings
    (seconds from the start of :meth:`Server.run`)."""

    job_id: int
    cfg: nc.NetConfig
    duration_ms: int
    arrival_s: float = 0.0
    footprint: int = 0           # estimated device bytes (admission)
    t_admit: Optional[float] = None
    t_start: Optional[float] = None   # built, first step queued
    t_done: Optional[float] = None
    steps_done: int = 0
    events: int = 0
    spikes: int = 0
    raster_sha256: str = ""
    device_bytes: int = 0        # held by its engine
    error: str = ""

    @property
    def latency_s(self) -> Optional[float]:
        return None if self.t_done is None else self.t_done - self.arrival_s

    @property
    def real_time_factor(self) -> Optional[float]:
        """Wall time from its first step to its completion per biological second."""
        if self.t_done is None or self.t_start is None:
            return None
        return (self.t_done - self.t_start) / (self.duration_ms * 1e-3)


def _real_engine(cfg, device):
    return E.Engine(cfg, device=device)


def _real_step_many(engines, n):
    E.step_many(engines, n)


class Server:
    """Continuous batching of simulation jobs on one GPU (see module doc).

    ``engine_factory(cfg, device)`` and ``step_many(engines, n)`` default to
    the engine; the host-side logic is tested on the CPU with stand-ins."""

    def __init__(self, device: int = 0, hbm_budget: float = 150e9, max_slots: int = 64, round_ms: int = 40,
                 build_workers: int = 8, engine_factory: Optional[Callable] = None,
                 step_many: Optional[Callable] = None):
        if not 1 <= round_ms <= 64:
            raise ValueError("round_ms must be in 1..64 (the engine keeps the spikes of its last 80 steps)")
        self.device = device
        self.hbm_budget = hbm_budget
        self.max_slots = max_slots
        self.round_ms = round_ms
        self.build_workers = build_workers
        self.engine_factory = engine_factory or _real_engine
        self.step_many = step_many or _real_step_many
        self.rounds = 0

    def run(self, jobs: List[Job], clock: Callable[[], float] = time.monotonic,
            idle_wait: Callable[[float], None] = time.sleep) -> List[Job]:
        """Serve ``jobs`` (their arrival_s offsets from now) to completion."""
        for j in jobs:
            if not j.footprint:
                j.footprint = estimate_device_bytes(j.cfg)
            if j.footprint > self.hbm_budget:
                j.error = f"footprint {j.footprint} B exceeds the budget {int(self.hbm_budget)} B"
        arrivals = collections.deque(sorted((j for j in jobs if not j.error), key=lambda j: j.arrival_s))
        queue = collections.deque()
        building = {}
        active = []           # (job, engine, digest)
        used = 0
        t0 = clock()
        pool = concurrent.futures.ThreadPoolExecutor(max_workers=self.build_workers)
        try:
            while arrivals or queue or building or active:
                now = clock() - t0
                while arrivals and arrivals[0].arrival_s <= now:
                    queue.append(arrivals.popleft())
                # admission: first come, first served, under slots and memory
                while queue and len(active) + len(building) < self.max_slots and \
                        used + queue[0].footprint <= self.hbm_budget:
                    j = queue.popleft()
                    j.t_admit = now
                    used += j.footprint
                    building[pool.submit(self.engine_factory, j.cfg, self.device)] = j
                for f in [f for f in building if f.done()]:
                    j = building.pop(f)
                    try:
                        eng = f.result()
                    except Exception as ex:   # a network the engine refuses
                        j.error = str(ex)
                        j.t_done = clock() - t0
                        used -= j.footprint
                        continue
                    j.t_start = clock() - t0
                    j.device_bytes = getattr(eng, "device_bytes", 0)
                    active.append((j, eng, hashlib.sha256()))
                if not active:
                    waits = [arrivals[0].arrival_s - now] if arrivals else []
                    if building:
                        waits.append(0.002)
                    if waits:
                        idle_wait(max(0.0, min(waits)))
                    continue
                # one round: the resident jobs advance together
                k = min(self.round_ms, min(j.duration_ms - j.steps_done for j, _, _ in active))
                self.step_many([e for _, e, _ in active], k)
                self.rounds += 1
                still = []
                for j, eng, h in active:
                    t_first = j.steps_done
                    ids, te, counts = eng.spikes_range(t_first, k)
                    o = 0
                    for c in counts:
                        c = int(c)
                        h.update(np.ascontiguousarray(ids[o:o + c], "<u4").tobytes())
                        h.update(np.ascontiguousarray(te[o:o + c], "<f8").tobytes())
                        o += c
                    j.spikes += len(ids)
                    j.steps_done += k
                    if j.steps_done >= j.duration_ms:
                        j.events = eng.events_delivered()
                        j.raster_sha256 = h.hexdigest()
                        eng.close()
                        j.t_done = clock() - t0
                        used -= j.footprint
                    else:
                        still.append((j, eng, h))
                active = still
        finally:
            for _, eng, _ in active:
                eng.close()
            for f in building:
                try:
                    f.result().close()
                except Exception:
                    pass
            pool.shutdown(wait=True)
        return jobs


def run_one_at_a_time(jobs: List[Job], device: int = 0, read_ms: int = 40,
                      clock: Callable[[], float] = time.monotonic) -> List[Job]:
    """The same jobs without the server: each built, stepped through its
    duration with dpsnn_step (its spikes read back every ``read_ms`` steps
    into the same raster digest) and released, one after another; times in
    seconds from the start."""
    t0 = clock()
    for j in jobs:
        j.t_admit = clock() - t0
        try:
            eng = E.Engine(j.cfg, device=device)
        except E.EngineError as ex:
            j.error = str(ex)
            j.t_done = clock() - t0
            continue
        j.t_start = clock() - t0
        j.device_bytes = eng.device_bytes
        h = hashlib.sha256()
        while j.steps_done < j.duration_ms:
            k = min(read_ms, j.duration_ms - j.steps_done)
            eng.step(k)
            ids, te, counts = eng.spikes_range(j.steps_done, k)
            o = 0
            for c in counts:
                c = int(c)
                h.update(np.ascontiguousarray(ids[o:o + c], "<u4").tobytes())
                h.update(np.ascontiguousarray(te[o:o + c], "<f8").tobytes())
                o += c
            j.spikes += len(ids)
            j.steps_done += k
        j.events = eng.events_delivered()
        j.raster_sha256 = h.hexdigest()
        eng.close()
        j.t_done = clock() - t0
    return jobs


def poisson_jobs(n_jobs: int, rate_per_s: float, seed: int = 7, max_side: int = 16,
                 duration_ms=(500, 10000), stdp_fraction: float = 0.2, nu_ext_hz=(1.0, 5.0)) -> List[Job]:
    """The served-simulations request stream: Poisson arrivals at
    ``rate_per_s``; grid side drawn log-uniformly from 1 to ``max_side``
    modules, biological duration uniform in ``duration_ms``, per-job seed and
    external rate, plasticity on for ``stdp_fraction`` of the jobs.  Each job
    is the run of one reference rank per cortical module (env_globH = the
    module count, at most the reference's 256 ranks), so that no emulated
    rank's serial bath stream is longer than one module.  Every job carries
    the delay-range sub-population: without it the reference refuses every
    grid of 6x6 modules and more, and a smaller one now and then (a delay
    level of 80 has a probability of 6e-8 per synapse); the engine refuses
    the same networks."""
    rng = np.random.default_rng(seed)
    t = 0.0
    jobs = []
    for i in range(n_jobs):
        t += rng.exponential(1.0 / rate_per_s)
        side = int(min(max_side, max(1, math.floor(math.exp(rng.uniform(0, math.log(max_side + 1)))))))
        dur = int(rng.integers(duration_ms[0], duration_ms[1] + 1))
        stdp = bool(rng.random() < stdp_fraction)
        cfg = nc.cortical_grid(side, side, total_ms=dur, seed=1 + i, nu_ext_hz=float(rng.uniform(*nu_ext_hz)),
                               stdp=stdp, start_plasticity_ms=0, delay_range_subpop=True,
                               glob_h=side * side, **({"p1": 0.0376} if side == 2 else {}))
        jobs.append(Job(job_id=i, cfg=cfg, duration_ms=dur, arrival_s=t))
    return jobs
