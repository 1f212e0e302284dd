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


# ---------------------------------------------------------------- summaries
# Networks too large to commit their raster are pinned by digests of it:
# per emission ms the spike count and a CRC-32 of that ms's spikes, per
# reference rank a SHA-256 of the rank's whole raster, and per sub-population
# firing rate and ISI coefficient of variation.  The canonical bytes of a set
# of spikes are its ids (uint32, little endian) then its emission times
# (float64), in ascending id order within a ms and time order within a rank,
# the order of the reference's per-rank spike files.

def summary(name):
    with np.load(os.path.join(HERE, f"{name}.summary.npz")) as z:
        return {k: z[k] for k in z.files}


def _canon(ids, ts):
    return np.ascontiguousarray(ids, dtype="<u4").tobytes() + np.ascontiguousarray(ts, dtype="<f8").tobytes()


def per_ms_digests(ids, ts, total_ms):
    """(count, crc32) per emission ms 0 .. total_ms-1 of a step-major raster
    (ascending id within each ms, as the engine and the reference emit it)."""
    import zlib
    ms = np.floor(ts).astype(np.int64)
    order = np.lexsort((ids, ms))
    ids, ts, ms = ids[order], ts[order], ms[order]
    edges = np.searchsorted(ms, np.arange(total_ms + 1))
    cnt = np.diff(edges).astype(np.int32)
    crc = np.zeros(total_ms, np.uint32)
    for m in range(total_ms):
        a, b = edges[m], edges[m + 1]
        crc[m] = zlib.crc32(_canon(ids[a:b], ts[a:b]))
    return cnt, crc


def rank_digests(ids, ts, glob_h, glob_n):
    """SHA-256 (32 bytes each) of every rank's raster, as a (glob_h, 32) uint8 array."""
    import hashlib
    loc = glob_n // glob_h
    rank = ids // loc
    o = np.lexsort((ids, ts, rank))   # per rank in time order, ties by id
    ids, ts, rank = ids[o], ts[o], rank[o]
    edges = np.searchsorted(rank, np.arange(glob_h + 1))
    out = np.zeros((glob_h, 32), np.uint8)
    for h in range(glob_h):
        a, b = edges[h], edges[h + 1]
        out[h] = np.frombuffer(hashlib.sha256(_canon(ids[a:b], ts[a:b])).digest(), np.uint8)
    return out


def pop_stats(ids, ts, counts, glob_n, t0_ms, t1_ms):
    """Per sub-population (``counts``: its neurons in one module) the mean
    firing rate in Hz over the emission window [t0_ms, t1_ms), and the ISI
    coefficient of variation: the mean, over the population's neurons with
    at least two inter-spike intervals in the window, of std(ISI)/mean(ISI).
    An empty population gives NaN for both."""
    npcm = int(sum(counts))
    n_mod = glob_n // npcm
    sel = (ts >= t0_ms) & (ts < t1_ms)
    ids, ts = ids[sel].astype(np.int64), ts[sel]
    o = np.lexsort((ts, ids))
    ids, ts = ids[o], ts[o]
    in_cm = ids % npcm
    bounds = np.cumsum([0] + list(counts))
    dur_s = (t1_ms - t0_ms) * 1e-3
    rates, cvs = [], []
    for s in range(len(counts)):
        if counts[s] == 0:
            rates.append(float("nan"))
            cvs.append(float("nan"))
            continue
        m = (in_cm >= bounds[s]) & (in_cm < bounds[s + 1])
        si, st = ids[m], ts[m]
        rates.append(len(si) / (counts[s] * n_mod * dur_s))
        same = si[1:] == si[:-1]
        isi = np.diff(st)[same]
        owner = si[1:][same]
        cv = []
        if len(isi):
            _, start, nisi = np.unique(owner, return_index=True, return_counts=True)
            for a, k in zip(start, nisi):
                if k >= 2:
                    x = isi[a:a + k]
                    cv.append(float(np.std(x) / np.mean(x)))
        cvs.append(float(np.mean(cv)) if cv else float("nan"))
    return rates, cvs
