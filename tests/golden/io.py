"""Readers of the committed golden fixtures."""
import gzip
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def manifest():
    with open(os.path.join(HERE, "manifest.json")) as f:
        return json.load(f)


def raster(name):
    """(ids, times) of the reference's full-precision raster, in file order."""
    ids, ts = [], []
    with gzip.open(os.path.join(HERE, f"{name}.raster.gz"), "rt") as f:
        for line in f:
            a, b = line.split()
            ids.append(int(a))
            ts.append(float(b))
    return np.array(ids, np.uint32), np.array(ts, np.float64)


def rank_major(ids, ts, glob_h, glob_n):
    """Reorder a step-major raster (every rank's spikes of a step, then the
    next step) into the order of the reference's per-rank files read one
    rank after the other."""
    rank = ids // (glob_n // glob_h)
    o = np.argsort(rank, kind="stable")
    return ids[o], ts[o]


def kat():
    out = {}
    with open(os.path.join(HERE, "ref_kat.txt")) as f:
        for line in f:
            name, i, v = line.split()
            out.setdefault(name, []).append(float.fromhex(v))
    return {k: np.array(v) for k, v in out.items()}


def raster_lines(ids, ts):
    """The %.17g raster text the reference writes, for comparison."""
    return "".join("%d %.17g\n" % (int(i), float(t)) for i, t in zip(ids, ts))
