"""Generate the golden fixtures of tests/golden from the reference itself.

Runs in the development container only (it needs the reference sources,
compiled by ``make -C oracle ref kat``); the fixtures it writes are committed
and are all the GPU box sees.  Each network is described by
``201812realtimecortsim_b200.netconfig`` and run with the reference binaries
built from the unmodified sources plus the bounds fix:

* ``ref_kat.txt``        ran3 / NormDev / Gaussian LUT / roundr2i values from
                          the reference's own randdev.o and erflib.o;
* ``<case>.raster.gz``   full-precision raster (%.17g) of the reference, rank
                          by rank when it runs several ranks (env_globH > 1,
                          one process per rank over oracle/mpi_shm);
* ``<case>.spikes.gz``   the reference's own spikes file (%.7g);
* ``manifest.json``      sha256 of the BACKWARD synapse dump and of the
                          output files (spikes, ratesPerPop,
                          FiringsInChronoWindow; with plasticity also the
                          synapse periodic probe files synPeriodicProbe_A/B
                          and the STDPevent files, from a run that enables
                          them),
                          spike and synaptic-event counts, configuration.

* ``<case>.summary.npz`` for the networks of ``SUMMARY_CASES``, whose
                          raster is too large to commit: per emission ms the
                          spike count and CRC-32, per rank the raster's
                          SHA-256 (see tests/golden/io.py), and per step the
                          synaptic events that raster delivers (with the
                          restatement's out-degree per neuron and delay);
                          their manifest
                          entry holds the BACKWARD dump SHA-256 of a few
                          ranks and the per-population firing rates and ISI
                          CV.  Those runs write the other ranks' synapse
                          dumps to /dev/null.

* the manifest entry of each network of ``REFUSED_CASES`` holds the first
  ERROR line the reference printed when it refused to build it.

Usage: python tests/golden/make_golden.py [case ...]
(with case names, only those entries of the manifest are regenerated)
"""
import gzip
import hashlib

import numpy as np
import importlib
import io
import json
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from tests.golden.cases import CASES, REFUSED_CASES, SUMMARY_CASES  # noqa: E402
from tests.golden import io as gio  # noqa: E402

nc = importlib.import_module("201812realtimecortsim_b200.netconfig")
REF_HP = os.path.join(ROOT, "oracle", "_ref", "dpsnn_ref_hp")
REF = os.path.join(ROOT, "oracle", "_ref", "dpsnn_ref")
# the same reference objects over the shared-memory MPI subset, for env_globH > 1
REF_MP_HP = os.path.join(ROOT, "oracle", "_ref", "dpsnn_ref_mp_hp")
REF_MP = os.path.join(ROOT, "oracle", "_ref", "dpsnn_ref_mp")
# built without -DDelayUniform: the reference Makefile's exponential delays
REF_EXP_HP = os.path.join(ROOT, "oracle", "_ref", "dpsnn_ref_exp_hp")
REF_EXP = os.path.join(ROOT, "oracle", "_ref", "dpsnn_ref_exp")
# the Perseo .ini writer switched on (compiled out of the stock build)
REF_INI = os.path.join(ROOT, "oracle", "_ref", "dpsnn_ref_ini")
KAT = os.path.join(ROOT, "oracle", "_ref", "ref_kat")
# the side outputs of a plasticity run: synapse probe and STDP event files
PROBE_ENV = {"env_statSynPeriodicProbe_writeDisable": "0", "env_startSynPeriodicProbe_s": "0",
             "env_stopSynPeriodicProbe_s": "100000", "env_statSTDPevent_writeDisable": "0",
             "env_startSTDPevent_s": "0", "env_stopSTDPevent_s": "100000"}


def sha256(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 20), b""):
            h.update(chunk)
    return h.hexdigest()


def gz_text(path):
    """Text writer of a gzip file with no timestamp (byte-stable output)."""
    return io.TextIOWrapper(gzip.GzipFile(path, "wb", mtime=0))


def run(binary, cfg, workdir, dump_ranks=None):
    env = dict(os.environ)
    env.update(cfg.write(workdir))
    if dump_ranks is not None:   # the other ranks' synapse dumps are not kept
        for h in range(cfg.glob_h):
            if h not in dump_ranks:
                os.symlink(os.devnull, os.path.join(
                    workdir, f"localNet_h{h}_N{cfg.glob_n // cfg.glob_h}_SynapticList_BACKWARD_R-1.dat"))
    if cfg.delay_exponential:
        binary = {REF_HP: REF_EXP_HP, REF: REF_EXP}[binary]
    if cfg.glob_h > 1:   # one process per rank
        binary = {REF_HP: REF_MP_HP, REF: REF_MP}[binary]
        env["DPSNN_SHM_RANKS"] = str(cfg.glob_h)
    r = subprocess.run([binary], cwd=workdir, env=env, capture_output=True, text=True)
    if r.returncode != 0 or "ERROR" in r.stdout:
        raise RuntimeError(r.stdout[-2000:] + r.stderr[-2000:])


def read_raster(hp, cfg):
    """The %.17g raster of every rank of a run, as (ids, times) arrays."""
    ids, ts = [], []
    for h in range(cfg.glob_h):
        for sec in range((cfg.total_ms + 999) // 1000):
            fn = os.path.join(hp, f"spikes-sec{sec}-C{cfg.n_modules}-H{cfg.glob_h}-h{h:03d}.dat")
            if os.path.exists(fn):
                a = np.loadtxt(fn, dtype=np.float64, ndmin=2)
                if a.size:
                    ids.append(a[:, 0].astype(np.uint32))
                    ts.append(a[:, 1])
    return np.concatenate(ids), np.concatenate(ts)


def make_summary(name, manifest):
    make, dump_ranks, (w0, w1) = SUMMARY_CASES[name]
    cfg = make()
    entry = {"total_ms": cfg.total_ms, "glob_h": cfg.glob_h, "glob_n": cfg.glob_n}
    with tempfile.TemporaryDirectory(dir=os.environ.get("DPSNN_GOLDEN_TMP")) as td:
        hp = os.path.join(td, "hp")
        os.makedirs(hp)
        run(REF_HP, cfg, hp, dump_ranks)
        entry["backward_sha256"] = {}
        for h in dump_ranks:
            fn = f"localNet_h{h}_N{cfg.glob_n // cfg.glob_h}_SynapticList_BACKWARD_R-1.dat"
            entry["backward_sha256"][str(h)] = sha256(os.path.join(hp, fn))
        ids, ts = read_raster(hp, cfg)
    cnt, crc = gio.per_ms_digests(ids, ts, cfg.total_ms)
    rd = gio.rank_digests(ids, ts, cfg.glob_h, cfg.glob_n)
    # synaptic events per step (addInputSpike calls, which the reference
    # does not print): the reference's raster over the out-degree per
    # (neuron, delay) of the restatement's generation
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import dpsnn_oracle as O
    ev = O.events_per_step(O.outdegree_by_delay(cfg), ids, ts, cfg.total_ms)
    np.savez_compressed(os.path.join(HERE, f"{name}.summary.npz"), count_per_ms=cnt, crc_per_ms=crc,
                        rank_sha256=rd, events_per_step=ev)
    rates, cvs = gio.pop_stats(ids, ts, [p.count for p in cfg.subpops], cfg.glob_n, w0, w1)
    entry.update({"spikes": int(len(ids)), "stats_window_ms": [w0, w1], "rates_hz": rates, "isi_cv": cvs})
    manifest[name] = entry
    print(name, len(ids), "spikes", rates, cvs, flush=True)


def make_refused(name, manifest):
    """Run a network the reference refuses; record its first ERROR line."""
    cfg = REFUSED_CASES[name]()
    with tempfile.TemporaryDirectory() as td:
        env = dict(os.environ)
        env.update(cfg.write(td))
        env["DPSNN_SHM_RANKS"] = str(cfg.glob_h)
        r = subprocess.run([REF_MP if cfg.glob_h > 1 else REF], cwd=td, env=env, capture_output=True, text=True)
    errors = [l for l in r.stdout.splitlines() if l.startswith("ERROR")]
    if not errors:
        raise RuntimeError(f"{name}: the reference did not refuse the network")
    manifest[name] = {"refused": errors[0], "glob_h": cfg.glob_h}
    print(name, errors[0], flush=True)


def main():
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref", "kat", "mp", "exp", "ini"], check=True,
                   capture_output=True)
    with open(os.path.join(HERE, "ref_kat.txt"), "w") as f:
        f.write(subprocess.run([KAT], check=True, capture_output=True, text=True).stdout)
    only = sys.argv[1:]
    manifest = {}
    if only:
        with open(os.path.join(HERE, "manifest.json")) as f:
            manifest = json.load(f)
    for name in SUMMARY_CASES:
        if only and name in only:
            make_summary(name, manifest)
    for name in REFUSED_CASES:
        if not only or name in only:
            make_refused(name, manifest)
    for name, make in CASES.items():
        if only and name not in only:
            continue
        cfg = make()
        entry = {"total_ms": cfg.total_ms, "glob_h": cfg.glob_h}
        with tempfile.TemporaryDirectory() as td:
            hp = os.path.join(td, "hp")
            run(REF_HP, cfg, hp)
            dump = [f for f in os.listdir(hp) if "SynapticList_BACKWARD" in f][0]
            entry["backward_dump"] = dump
            entry["backward_sha256"] = sha256(os.path.join(hp, dump))
            lines = []   # rank-major: all of rank 0's lines, then rank 1's, ...
            for h in range(cfg.glob_h):
                for sec in range((cfg.total_ms + 999) // 1000):
                    fn = os.path.join(hp, f"spikes-sec{sec}-C{cfg.n_modules}-H{cfg.glob_h}-h{h:03d}.dat")
                    if os.path.exists(fn):
                        with open(fn) as f:
                            lines += f.readlines()
            entry["spikes"] = len(lines)
            with gz_text(os.path.join(HERE, f"{name}.raster.gz")) as f:
                f.writelines(lines)
            std = os.path.join(td, "std")
            run(REF, cfg, std)
            outs = {}
            for fn in sorted(os.listdir(std)):
                if fn.startswith(("spikes-", "ratesPerPop-", "FiringsInChronoWindow_")):
                    outs[fn] = sha256(os.path.join(std, fn))
            entry["outputs_sha256"] = outs
            with gz_text(os.path.join(HERE, f"{name}.spikes.gz")) as f:
                for h in range(cfg.glob_h):
                    with open(os.path.join(std, f"spikes-sec0-C{cfg.n_modules}-H{cfg.glob_h}-h{h:03d}.dat")) as g:
                        f.write(g.read())
            if cfg.stdp is not None:
                pr = os.path.join(td, "probe")
                probe = make()
                probe.extra_env.update(PROBE_ENV)
                run(REF, probe, pr)
                entry["probe_sha256"] = {fn: sha256(os.path.join(pr, fn)) for fn in sorted(os.listdir(pr))
                                         if fn.startswith("synPeriodicProbe_")}
                entry["stdp_event_sha256"] = {fn: sha256(os.path.join(pr, fn)) for fn in sorted(os.listdir(pr))
                                              if fn.startswith("STDPevent-")}
            if cfg.glob_h == 1 and not cfg.delay_exponential:
                ini = os.path.join(td, "ini")
                short = make()
                short.total_ms = 10   # the files are written at init
                run(REF_INI, short, ini)
                entry["ini_sha256"] = {fn: sha256(os.path.join(ini, fn)) for fn in sorted(os.listdir(ini))
                                       if fn.startswith(("PerseoConFile_", "PerseoModFile_"))}
        # synaptic events delivered in the run (identical dynamics in the
        # restatement, pinned by the raster and dump checks)
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import dpsnn_oracle as O
        net = O.OracleNet(cfg)
        ev = 0
        for _ in range(cfg.total_ms):
            net.step()
            ev += net.last_event_count()
        entry["events"] = ev
        manifest[name] = entry
        print(name, entry["spikes"], "spikes", flush=True)
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
