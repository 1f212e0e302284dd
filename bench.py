"""Benchmark: synaptic events/s of DPSNN's per-timestep loop on the 24x24 grid.

One bench step is one 1 ms simulation step of the 24x24 cortical-module grid
(720000 neurons, ~0.81 G synapses, 10 s network; STDP off) -- synapse
delivery, Poisson bath, LIFCA update and spike compaction for the whole grid,
with the RNG streams of 192 reference ranks (env_globH=192, the largest
reference decomposition of this grid: 3 modules per rank).  The network lives
in HBM; the timed region covers K consecutive steps after W warm-up steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

value  = synaptic events delivered in the K steps / device time (CUDA events
         on the engine stream), summed over ranks (independent replicas).
e2e    = the same metric through the C ABI as a drop-in caller uses it: one
         dpsnn_step per ms and the step's spike list read back to host memory
         (the raster), timed on the host; no per-step input goes to the device.
--batch J runs the batched sweep instead: J independent networks of 1x1-4x4
modules, --batch-ms biological ms of each, one after another (dpsnn_step),
together (dpsnn_step_many) and together in autotuned CUDA graphs of 80 steps,
printing one JSON line with the three aggregate rates.
The reference arm (--impl reference) runs the reference built from its
sources on the same network and steps as the engine's timed region, as 192
MPI processes (a forked shared-memory MPI subset, oracle/mpi_shm) on the
host cores, timed by its own per-step chrono over steps W..W+K-1.
"""
from __future__ import annotations

import argparse
import concurrent.futures
import importlib
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "synaptic events/s"
UNIT = "events/s"
WORKLOAD = "24x24 grid, 720000 neurons, ~0.81G synapses, 1 ms steps, STDP off, RNG streams of 192 ranks"


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.out,
                stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        self.out.flush()
        self.out.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl" if args.impl == "b200" else "gloo",
                                timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


FIRE_RE = re.compile(r"total fire time = ([0-9.eE+-]+)")


def reference_c1_start(workdir: str, binary: str):
    """Start the reference binary on the 2x2 grid (1000 ms, 1 rank) in
    ``workdir``; the caller waits and parses its output."""
    nc = importlib.import_module("201812realtimecortsim_b200.netconfig")
    cfg = nc.cortical_grid(2, 2, total_ms=1000)
    os.makedirs(workdir, exist_ok=True)
    env = dict(os.environ)
    env.update(cfg.write(workdir))
    # the reference's own switches for its raster and rate files: off, so
    # that its timed loop does no file output (the engine's loop does none)
    env["env_spikes_writeDisable"] = "1"
    env["env_statRatesPerPop_writeDisable"] = "1"
    # its 185 MB synapse-list text dump at init goes to /dev/null
    os.symlink(os.devnull, os.path.join(workdir, f"localNet_h0_N{cfg.glob_n}_SynapticList_BACKWARD_R-1.dat"))
    return subprocess.Popen([binary], cwd=workdir, env=env, stdout=subprocess.PIPE,
                            stderr=subprocess.DEVNULL, text=True)


def reference_fire_seconds(proc) -> float:
    """Time the reference spent in localNetProcess_fire (its own CHRONO line:
    the 1001 simulation steps, connectome construction excluded)."""
    out, _ = proc.communicate()
    if proc.returncode != 0:
        raise RuntimeError("reference run failed")
    m = FIRE_RE.search(out)
    if not m:
        raise RuntimeError("reference output has no fire time")
    return float(m.group(1))


def reference_events_c1() -> int:
    with open(os.path.join(ROOT, "tests", "golden", "manifest.json")) as f:
        return int(json.load(f)["c1_2x2"]["events"])


def bench_network(args):
    """The benchmark network (netconfig) and its workload name.  The grid
    carries the empty delay-range sub-population, without which the
    reference refuses networks of this size (netconfig.cortical_grid)."""
    nc = importlib.import_module("201812realtimecortsim_b200.netconfig")
    cfx, cfy = (int(x) for x in args.grid.lower().split("x"))
    total_ms = max(args.full_ms, args.warmup + args.steps + 10)
    cfg = nc.cortical_grid(cfx, cfy, total_ms=total_ms, glob_h=args.ranks, delay_range_subpop=True,
                           stdp=args.stdp, start_plasticity_ms=0)
    if args.stdp:
        workload = (f"{cfx}x{cfy} grid, {cfg.glob_n} neurons, 1 ms steps, pair-based additive STDP on E->E "
                    f"synapses from t=0 (A+ 0.01, A- 0.012, tau 20 ms, weights in [0, 2 mu], updated each s), "
                    f"RNG streams of {args.ranks} ranks")
    elif (cfx, cfy, args.ranks) == (24, 24, 192):
        workload = WORKLOAD
    else:
        workload = f"{cfx}x{cfy} grid, {cfg.glob_n} neurons, 1 ms steps, STDP off, RNG streams of {args.ranks} ranks"
    return cfg, workload


PARTIAL_RE = re.compile(r"PartialTimeStep = ([0-9.eE+-]+)")
REF_CASE = "c2_24x24_p192"   # reference-derived events per step of the benchmark network


def reference_window(cfg, binary, workdir, W, K, raster):
    """Run the reference (env_globH processes over oracle/mpi_shm) for W+K
    steps of ``cfg`` in ``workdir``; return the seconds its own
    PartialTimeStep chrono (DPSNN_localNet_sim.c:59,305) measured over steps
    W..W+K-1, the slowest rank's.  Without ``raster`` its spike and rate
    files are off (its fastest stock configuration); its synapse-list dump
    goes to /dev/null."""
    os.makedirs(workdir, exist_ok=True)
    env = dict(os.environ)
    env.update(cfg.write(workdir))
    env["env_totalSimTime_ms"] = str(W + K)
    env["env_startPartialChrono_ms"] = str(W)
    env["env_partialChronoWindow_ms"] = str(K)
    if not raster:
        env["env_spikes_writeDisable"] = "1"
        env["env_statRatesPerPop_writeDisable"] = "1"
    env["DPSNN_SHM_RANKS"] = str(cfg.glob_h)
    os.symlink(os.devnull, os.path.join(
        workdir, f"localNet_h0_N{cfg.glob_n // cfg.glob_h}_SynapticList_BACKWARD_R-1.dat"))
    r = subprocess.run([binary], cwd=workdir, env=env, capture_output=True, text=True)
    if r.returncode != 0 or "ERROR" in r.stdout:
        raise RuntimeError("reference run failed: " + (r.stdout[-500:] + r.stderr[-500:]).strip())
    secs = []
    for h in range(cfg.glob_h):
        with open(os.path.join(workdir, f"SummaryStatMeasures_h{h}.stat")) as f:
            m = PARTIAL_RE.search(f.read())
        if not m:
            raise RuntimeError(f"rank {h} reported no PartialTimeStep")
        secs.append(float(m.group(1)))
    return max(secs)


def reference_window_events(cfg, W, K, workdir):
    """Synaptic events of steps W..W+K-1 (addInputSpike calls; the reference
    prints no count): the committed reference-derived counts of the
    benchmark network, else those of an untimed full-precision reference run
    over the restatement's out-degree per (neuron, delay)."""
    man = os.path.join(ROOT, "tests", "golden", "manifest.json")
    npz = os.path.join(ROOT, "tests", "golden", f"{REF_CASE}.summary.npz")
    if os.path.exists(npz):
        sys.path.insert(0, ROOT)
        from tests.golden.cases import SUMMARY_CASES
        ref_cfg = SUMMARY_CASES[REF_CASE][0]()
        same = (ref_cfg.env() | {"env_totalSimTime_ms": "", "env_partialChronoWindow_ms": ""}) == \
               (cfg.env() | {"env_totalSimTime_ms": "", "env_partialChronoWindow_ms": ""}) and \
               ref_cfg.column_txt() == cfg.column_txt() and ref_cfg.connectivity_txt() == cfg.connectivity_txt()
        import numpy as np
        ev = []
        if same:
            with np.load(npz) as z:
                ev = z["events_per_step"]
        if same and W + K <= len(ev):
            return int(ev[W:W + K].sum()), "reference raster of the benchmark network (tests/golden), " \
                                            "restatement out-degree"
    binary = os.path.join(ROOT, "oracle", "_ref", "dpsnn_ref_mp_hp" if cfg.glob_h > 1 else "dpsnn_ref_hp")
    reference_window(cfg, binary, workdir, W, K, raster=True)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import dpsnn_oracle as O
    import numpy as np
    ids, ts = [], []
    for h in range(cfg.glob_h):
        fn = os.path.join(workdir, f"spikes-sec0-C{cfg.n_modules}-H{cfg.glob_h}-h{h:03d}.dat")
        if os.path.exists(fn) and os.path.getsize(fn):
            a = np.loadtxt(fn, ndmin=2)
            ids.append(a[:, 0].astype(np.int64))
            ts.append(a[:, 1])
    ids = np.concatenate(ids) if ids else np.zeros(0, np.int64)
    ts = np.concatenate(ts) if ts else np.zeros(0)
    ev = O.events_per_step(O.outdegree_by_delay(cfg), ids, ts, W + K)
    return int(ev[W:W + K].sum()), "untimed full-precision reference run, restatement out-degree"


def run_reference(args, world, rank):
    """Reference arm: the reference built from its sources, on the same
    network and steps as the engine's timed region (steps W..W+K-1), run as
    env_globH MPI processes (oracle/mpi_shm: forked processes over shared
    memory) on the host cores; time = its own PartialTimeStep chrono over
    those steps."""
    if rank != 0:
        return
    cfg, workload = bench_network(args)
    W, K = args.warmup, args.steps
    binary = os.path.join(ROOT, "oracle", "_ref", "dpsnn_ref_mp" if cfg.glob_h > 1 else "dpsnn_ref")
    if not os.path.exists(binary):
        print(json.dumps({"impl": "reference", "unavailable": f"{os.path.relpath(binary, ROOT)} was not built"}))
        return
    need_gb = 0.3 * cfg.glob_h * (cfg.glob_n / cfg.glob_h) / 3750.0   # ~0.21 GB per rank of 3750 neurons
    try:
        import psutil
        avail_gb = psutil.virtual_memory().available / 1e9
    except Exception:
        avail_gb = need_gb
    if avail_gb < need_gb:
        print(json.dumps({"impl": "reference", "unavailable": f"{cfg.glob_h} reference processes need "
                          f"~{need_gb:.0f} GB of host memory, {avail_gb:.0f} GB available"}))
        return
    with tempfile.TemporaryDirectory() as td:
        secs = reference_window(cfg, binary, os.path.join(td, "timed"), W, K, raster=False)
        events, how = reference_window_events(cfg, W, K, os.path.join(td, "events"))
    value = events / secs
    cores = min(cfg.glob_h, os.cpu_count() or 1)   # one process per rank, at most one per host thread busy
    sample = (f"reference built from its sources, {workload}, steps {W}-{W + K - 1}, {cfg.glob_h} MPI "
              f"processes on {cores} host threads, spike and rate files off; time = its PartialTimeStep "
              f"chrono (slowest rank), {secs:.3f} s; events: {how}")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": K, "warmup": W, "ms_per_step": 1e3 * secs / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: network generated by the reference's own generator, seed 1",
        "config": {"workload": workload, "parallelism": f"{cfg.glob_h} MPI processes",
                   "real_time_factor": secs / (K * 1e-3), "events_per_step": events / K,
                   "timed_steps": [W, W + K - 1]},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_batch(args):
    """One JSON line for the batched form: the same jobs (batch.sweep_configs)
    on freshly built engines in three arms, each timed over steps 1..K after
    an untimed first step (K = --batch-ms rounded up to a multiple of 80):
      sequential -- one job after another, dpsnn_step;
      step_many  -- all jobs together, dpsnn_step_many (one step of every
                    job at a time, their kernels overlapping);
      graph      -- all jobs together in CUDA graphs of 80 steps, with the
                    launch shapes the autotuner picked (tuned untimed on the
                    step_many arm's engines after their timed region).
    Host wall time between device synchronisations (the arms span many
    streams); each arm's per-job event counts must be identical."""
    import torch
    E = importlib.import_module("201812realtimecortsim_b200.engine")
    B = importlib.import_module("201812realtimecortsim_b200.batch")
    K = -(-max(args.batch_ms, 1) // B.GRAPH_STEPS) * B.GRAPH_STEPS
    tune_steps = len(B.CANDIDATES) * 2 * B.GRAPH_STEPS
    jobs = B.sweep_configs(args.batch, total_ms=K + tune_steps + 10)
    sync = torch.cuda.synchronize
    res, build_s, extra = {}, {}, {}
    best_rule = None
    for arm in ("sequential", "step_many", "graph"):
        tb0 = time.perf_counter()
        engines = B.build_all(jobs, threads=16)
        sync()
        build_s[arm] = time.perf_counter() - tb0
        if arm == "graph":
            for e, c in zip(engines, jobs):
                e.set_launch_shape(*best_rule(e, c))
        E.step_many(engines, 1)
        for e in engines:
            e.sync()
        ev0 = [e.events_delivered() for e in engines]
        runner = None
        if arm == "graph":
            tg = time.perf_counter()
            runner = B.BatchRunner(engines)
            extra["graph_record_s"] = time.perf_counter() - tg
        sync()
        t0 = time.perf_counter()
        if arm == "sequential":
            for e in engines:
                e.step(K)
                e.sync()
        elif arm == "step_many":
            E.step_many(engines, K)
        else:
            runner.run(K)
        for e in engines:
            e.sync()
        sync()
        dt = time.perf_counter() - t0
        ev = [e.events_delivered() - a for e, a in zip(engines, ev0)]
        res[arm] = (dt, ev)
        print(f"[batch] {arm}: {K} steps of {len(jobs)} networks in {dt:.3f} s", file=sys.stderr, flush=True)
        if runner is not None:
            runner.close()
        if arm == "step_many":
            tune = B.autotune(engines, jobs, sync)
            best_rule = B.shape_rule(tune["blocks_per_module"])
            extra["autotune"] = {"blocks_per_module": tune["blocks_per_module"],
                                 "seconds_per_graph_run": {str(k): v for k, v in tune["seconds"].items()}}
        for e in engines:
            e.close()
        del engines
    neurons = sum(c.glob_n for c in jobs)
    evs = res["sequential"][1]
    print(json.dumps({
        "metric": "aggregate synaptic events/s (batched sweep)", "value": sum(res["graph"][1]) / res["graph"][0],
        "unit": UNIT, "n_gpus": 1, "higher_is_better": True, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{len(jobs)} independent networks of 1x1-4x4 modules ({neurons} neurons), "
                               f"steps 1..{K} of each, per-job seed, NuExt 1-5 Hz, AlphaC 0-2, STDP off, "
                               f"one emulated rank per module",
                   "timing": "host wall time between device synchronisations"},
        "seconds": {a: r[0] for a, r in res.items()},
        "values": {a: sum(r[1]) / r[0] for a, r in res.items()},
        "build_s": build_s, **extra,
        "per_job_events_identical": all(r[1] == evs for r in res.values()),
    }), flush=True)


def run_serve(args):
    """The served form (continuous batching) against the same jobs one at a
    time: J jobs of the served-simulations stream (Poisson arrivals at 50/s,
    1x1-16x16 modules log-uniform, 0.5-10 s of biological time scaled by
    --serve-scale, 20 % with plasticity) under a 150 GB device-memory budget;
    each arm on the same GPU, host wall time from the first arrival to the
    last completion (builds included)."""
    import numpy as np
    S = importlib.import_module("201812realtimecortsim_b200.serve")

    def stream():
        jobs = S.poisson_jobs(args.serve, rate_per_s=50.0, seed=11)
        for j in jobs:
            j.duration_ms = max(1, int(round(j.duration_ms * args.serve_scale)))
            j.cfg.total_ms = j.duration_ms + 1
        return jobs

    served = stream()
    srv = S.Server(device=0, hbm_budget=150e9, max_slots=args.serve_slots, round_ms=40)
    t0 = time.perf_counter()
    srv.run(served)
    t_served = time.perf_counter() - t0
    # the same jobs one at a time: build, dpsnn_step through the duration
    # with the spikes read back every 40 steps, release
    alone = stream()
    t0 = time.perf_counter()
    S.run_one_at_a_time(alone, device=0, read_ms=40)
    t_alone = time.perf_counter() - t0
    ok = [j for j in served if not j.error]
    lat = np.array([j.latency_s for j in ok])
    rtf = np.array([j.real_time_factor for j in ok])
    ev_s = sum(j.events for j in ok)
    ev_a = sum(j.events for j in alone if not j.error)
    print(json.dumps({
        "metric": "aggregate synaptic events/s (served jobs)", "value": ev_s / t_served, "unit": UNIT,
        "n_gpus": 1, "higher_is_better": True, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{len(served)} jobs: Poisson arrivals at 50/s, 1x1-16x16 modules (log-uniform), "
                               f"0.5-10 s x {args.serve_scale} of biological time, 20% with STDP, one emulated "
                               f"rank per module, 150 GB budget, {args.serve_slots} slots",
                   "timing": "host wall time from the first arrival to the last completion, builds included"},
        "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                      "max": float(lat.max())},
        "real_time_factor": {"p50": float(np.percentile(rtf, 50)), "p99": float(np.percentile(rtf, 99))},
        "served_s": t_served, "one_at_a_time_s": t_alone, "one_at_a_time_value": ev_a / t_alone,
        "ratio_vs_one_at_a_time": (ev_s / t_served) / (ev_a / t_alone) if ev_a else None,
        "results_identical_to_one_at_a_time": all(a.raster_sha256 == b.raster_sha256 and a.events == b.events
                                                   for a, b in zip(served, alone) if not a.error),
        "refused": [j.error for j in served if j.error],
        "rounds": srv.rounds,
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--e2e-steps", type=int, default=0, help="0 = the same K steps as the timed region")
    ap.add_argument("--full-ms", type=int, default=10000,
                    help="steps of the whole run timed for full_run (the network's biological ms; 0 = skip)")
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--grid", default="24x24", help="CFXxCFY modules (profiling of smaller grids)")
    ap.add_argument("--ranks", type=int, default=192, help="env_globH: emulated reference ranks")
    ap.add_argument("--stdp", action="store_true",
                    help="plasticity on (the 48x48 configuration: --grid 48x48 --ranks 256 --stdp)")
    ap.add_argument("--batch", type=int, default=0, help="run the batched sweep of this many networks instead")
    ap.add_argument("--serve", type=int, default=0, help="run the served form with this many jobs instead")
    ap.add_argument("--serve-scale", type=float, default=0.1,
                    help="scale of the jobs' biological durations (a bounded sample)")
    ap.add_argument("--serve-slots", type=int, default=64, help="jobs resident at once")
    ap.add_argument("--batch-ms", type=int, default=100,
                    help="biological ms per network timed in the batched sweep (a bounded sample)")
    args = ap.parse_args()
    if args.batch:
        run_batch(args)
        return
    if args.serve:
        run_serve(args)
        return
    args.warmup = max(args.warmup, 3)
    world, rank, local, dist = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    import torch
    E = importlib.import_module("201812realtimecortsim_b200.engine")
    torch.cuda.set_device(local)
    cfg, workload = bench_network(args)
    total_ms = cfg.total_ms

    def all_max(x):
        if not dist:
            return x
        t = torch.tensor([float(x)], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def all_sum(x):
        if not dist:
            return x
        t = torch.tensor([float(x)], device="cuda", dtype=torch.float64)
        dist.all_reduce(t)
        return float(t.item())

    def device_seconds(eng, stream, n):
        """Device time of n steps on the engine stream (CUDA events)."""
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        eng.step(n)
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b) * 1e-3

    # 1. timed region: steps W .. W+K-1, device time on the engine stream
    eng = E.Engine(cfg, device=local)
    eng_bytes = 6 * eng.synapse_count
    stream = torch.cuda.ExternalStream(eng.cuda_stream())
    warm_s = device_seconds(eng, stream, args.warmup)
    eng.sync()
    e0 = eng.events_delivered()
    l0 = eng.kernel_launches()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        elapsed = device_seconds(eng, stream, args.steps)
    torch.cuda.synchronize()
    eng.sync()
    events = eng.events_delivered() - e0
    launches = eng.kernel_launches() - l0
    t_max = all_max(elapsed)
    ev_tot = all_sum(events)

    # 2. the whole run the metric is quoted on (the network's total_ms steps,
    # 10 s by default): the same engine continues; device time of its three
    # segments (warm-up, timed region, the rest)
    full = None
    rest = total_ms - args.warmup - args.steps
    if args.full_ms and rest > 0:
        with ClockSampler(local) as clk_full:
            rest_s = device_seconds(eng, stream, rest)
        eng.sync()
        full_s = all_max(warm_s + elapsed + rest_s)
        full_ev = all_sum(eng.events_delivered())
        full = {"steps": total_ms, "seconds": full_s, "real_time_factor": full_s / (total_ms * 1e-3),
                "value": full_ev / full_s, "unit": UNIT, "events_per_step": full_ev / world / total_ms,
                "clocks": clk_full.summary()}
    eng.close()

    # 3. per-kernel-family device times on an identical replay of steps
    # W .. W+K-1 (the simulation is deterministic: same network, same
    # steps); event pairs around each family, kept out of the timed region
    eng = E.Engine(cfg, device=local)
    eng.step(args.warmup)
    eng.sync()
    p0 = eng.events_delivered()
    eng.set_timing(True)
    eng.step(args.steps)
    eng.sync()
    eng.set_timing(False)
    ksec, kcnt = eng.kernel_times()
    prof_events = eng.events_delivered() - p0
    eng.close()

    # 4. e2e: the same steps W..W+K-1 of the same network, stepped one at a
    # time through the C ABI with each step's spike list read back to host
    # memory, timed on the host
    eng = E.Engine(cfg, device=local)
    eng.step(args.warmup)
    eng.sync()
    e2e_steps = args.steps if args.e2e_steps <= 0 else min(args.e2e_steps, args.steps)
    d2h = 0
    ee0 = eng.events_delivered()
    if dist:
        dist.barrier()
    h0 = time.perf_counter()
    for k in range(e2e_steps):
        eng.step(1)
        ids, te = eng.spikes(args.warmup + k)
        d2h += ids.nbytes + te.nbytes + 8   # + error flags and count
    eng.sync()   # the last step's remaining kernels are inside the timed region too
    h1 = time.perf_counter()
    e2e_events = eng.events_delivered() - ee0
    e2e_val = all_sum(e2e_events) / all_max(h1 - h0)
    eng.close()

    hbm, peak_kind = peaks()
    fam = E.TIMING_NAMES
    fam_total = float(sum(ksec)) or 1.0
    kernel_share = {f: float(s) / fam_total for f, s in zip(fam, ksec)}
    kernel_ms = {f: (1e3 * float(s) / args.steps) for f, s in zip(fam, ksec)}   # per step
    # delivery kernel: per synaptic event it reads the u32 target and the
    # i16 weight of the synapse and writes one 8-byte {key, weight} record
    deliver_s = float(ksec[1]) / max(int(kcnt[1]), 1)
    ev_per_launch = prof_events / max(int(kcnt[1]), 1)
    achieved = 14.0 * ev_per_launch / deliver_s / 1e9 if deliver_s > 0 else 0.0
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "deliver_traffic.json")
    if os.path.exists(tfile):
        with open(tfile) as f:
            traffic = float(json.load(f)["dram_bytes_per_event"]) * ev_per_launch
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        binary = os.path.join(ROOT, "oracle", "_ref", "dpsnn_ref")
        if os.path.exists(binary):
            with tempfile.TemporaryDirectory() as td:
                fire = reference_fire_seconds(reference_c1_start(td, binary))
            cpu = {"value": reference_events_c1() / fire, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": f"reference binary, 2x2 grid (5000 neurons, 5.6M synapses), 1000 ms, 1 rank, "
                             f"{fire:.1f} s in fire()"}
    if rank == 0:
        clocks = clk.summary()
        out = {
            "metric": METRIC, "value": ev_tot / t_max, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: network generated by the reference's algorithm, seed 1",
            "config": {"workload": workload, "global_batch": world, "seq_len": args.steps,
                       "parallelism": f"replicas x{world}",
                       "l2": f"inputs larger than L2 (connectome {eng_bytes / 1e9:.1f} GB of CSR read every step)",
                       "real_time_factor": t_max / (args.steps * 1e-3),
                       "events_per_step": events / args.steps,
                       "timed_steps": [args.warmup, args.warmup + args.steps - 1]},
            "roofline": {"bound": "hbm", "kernel": "deliver_kernel", "achieved": achieved, "peak": hbm,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": traffic, "algorithmic_bytes_per_event": 14,
                         "events_per_launch": ev_per_launch},
            "kernel_ms_per_step": kernel_ms,
            "kernel_share": kernel_share,
            "kernel_replay": {"steps": [args.warmup, args.warmup + args.steps - 1],
                              "events_identical_to_timed": prof_events == events},
            "full_run": full,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": d2h / max(e2e_steps, 1), "steps": e2e_steps,
                    "ms_per_step": 1e3 * (h1 - h0) / max(e2e_steps, 1)},
            "gpu_launches": launches,
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()

if __name__ == "__main__":
    main()
