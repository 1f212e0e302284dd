"""ctypes binding of the CPU restatement (dpsnn_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libdpsnn_oracle.so")
REF_BIN = os.path.join(HERE, "_ref", "dpsnn_ref")
REF_BIN_HP = os.path.join(HERE, "_ref", "dpsnn_ref_hp")

MAX_SUB = 27
MAX_ST = 8


class DpoConfig(C.Structure):
    _fields_ = [
        ("cfx", C.c_uint32), ("cfy", C.c_uint32), ("nsub", C.c_uint32),
        ("count", C.c_uint32 * MAX_SUB),
        ("JExt", C.c_float * MAX_SUB), ("DJExt", C.c_float * MAX_SUB), ("NuExt", C.c_float * MAX_SUB),
        ("Tau", C.c_float * MAX_SUB), ("Theta", C.c_float * MAX_SUB), ("H", C.c_float * MAX_SUB),
        ("Tarp", C.c_float * MAX_SUB), ("AlphaC", C.c_float * MAX_SUB), ("TauC", C.c_float * MAX_SUB),
        ("gC", C.c_float * MAX_SUB),
        ("J", (C.c_float * MAX_SUB) * MAX_SUB), ("DJ", (C.c_float * MAX_SUB) * MAX_SUB),
        ("DMin", (C.c_float * MAX_SUB) * MAX_SUB), ("DMax", (C.c_float * MAX_SUB) * MAX_SUB),
        ("spec", (((C.c_float * MAX_ST) * MAX_ST) * MAX_SUB) * MAX_SUB),
        ("stencil_dim", C.c_uint32),
        ("bath", (C.c_uint32 * MAX_ST) * MAX_ST),
        ("D", C.c_uint32), ("glob_h", C.c_uint32), ("global_seed", C.c_uint32),
        ("start_plasticity_ms", C.c_uint32), ("stop_plasticity_ms", C.c_uint32),
        ("min_syn_weight_f", C.c_float),
        ("stdp_antiCausalCoeff", C.c_float), ("stdp_multiplier", C.c_float),
        ("stdp_tau_ms", C.c_float), ("stdp_causalMax", C.c_float),
        ("stdp_antiCausalMax", C.c_float), ("stdp_tauDecay_s", C.c_float),
        ("stdp_drift", C.c_float),
        ("delay_exp", C.c_uint32),
    ]


def _lib():
    if not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", HERE, "port"], check=True, capture_output=True)
    lib = C.CDLL(LIB_PATH)
    P = C.c_void_p
    lib.dpo_create.restype = P
    lib.dpo_create.argtypes = [C.POINTER(DpoConfig), C.c_int]
    lib.dpo_destroy.argtypes = [P]
    lib.dpo_outdegree_by_delay.argtypes = [C.POINTER(DpoConfig), C.c_int, P]
    lib.dpo_last_error.restype = C.c_char_p
    for name in ("dpo_glob_n", "dpo_loc_n", "dpo_time_ms"):
        getattr(lib, name).restype = C.c_uint32
        getattr(lib, name).argtypes = [P]
    for name in ("dpo_total_synapses", "dpo_last_event_count", "dpo_last_bath_count"):
        getattr(lib, name).restype = C.c_uint64
        getattr(lib, name).argtypes = [P]
    lib.dpo_rank_synapse_count.restype = C.c_uint64
    lib.dpo_rank_synapse_count.argtypes = [P, C.c_uint32]
    lib.dpo_rank_synapses.argtypes = [P, C.c_uint32] + [P] * 5
    lib.dpo_rank_plasticity.argtypes = [P, C.c_uint32, P, P]
    lib.dpo_bath_params.argtypes = [P, P, P]
    lib.dpo_bath_lut.argtypes = [P, C.c_uint32, P]
    lib.dpo_write_backward_dump.argtypes = [P, C.c_char_p]
    lib.dpo_step.restype = C.c_int64
    lib.dpo_step.argtypes = [P]
    lib.dpo_last_spikes.argtypes = [P, P, P]
    lib.dpo_state.argtypes = [P] * 6
    lib.dpo_ran3_sequence.argtypes = [C.c_int32, C.c_uint32, P]
    lib.dpo_normdev_sequence.argtypes = [C.c_int32, C.c_uint32, P]
    lib.dpo_gaussian_lut.argtypes = [C.c_double] * 4 + [P]
    lib.dpo_roundr2i.restype = C.c_uint32
    lib.dpo_roundr2i.argtypes = [C.c_double]
    lib.dpo_exp_cr.restype = C.c_double
    lib.dpo_exp_cr.argtypes = [C.c_double]
    lib.dpo_log_cr.restype = C.c_double
    lib.dpo_log_cr.argtypes = [C.c_double]
    return lib


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        _LIB = _lib()
    return _LIB


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def config_from_netconfig(cfg) -> DpoConfig:
    """Fill the restatement's config from a ``netconfig.NetConfig``."""
    c = DpoConfig()
    c.cfx, c.cfy, c.nsub = cfg.cfx, cfg.cfy, len(cfg.subpops)
    for i, p in enumerate(cfg.subpops):
        c.count[i] = p.count
        for f in ("JExt", "DJExt", "NuExt", "Tau", "Theta", "H", "Tarp", "AlphaC", "TauC", "gC"):
            getattr(c, f)[i] = float(np.float32(getattr(p, f)))
    S = cfg.stencil_dim
    for (s, t), (J, DJ, dmin, dmax, probs) in cfg.conn.items():
        c.J[s][t] = float(np.float32(J))
        c.DJ[s][t] = float(np.float32(DJ))
        c.DMin[s][t] = float(np.float32(dmin))
        c.DMax[s][t] = float(np.float32(dmax))
        for y in range(S):
            for x in range(S):
                c.spec[s][t][x][y] = float(np.float32(probs[y * S + x]))
    c.stencil_dim = S
    for x in range(S):
        for y in range(S):
            c.bath[x][y] = cfg.bath_cext
    c.D, c.glob_h, c.global_seed = cfg.D, cfg.glob_h, cfg.seed
    c.start_plasticity_ms, c.stop_plasticity_ms = cfg.start_plasticity_ms, cfg.stop_plasticity_ms
    c.min_syn_weight_f = float(np.float32(cfg.min_syn_weight_f))
    if cfg.stdp is not None:
        _, anti, mult, tau, cmax, amax, tdec, drift = cfg.stdp
    else:   # readPlasticityParametersFile defaults
        anti, mult, tau, cmax, amax, tdec, drift = -1.0, 0.001, 20.0, 0.1, 0.12, 1.0, 0.0
    c.stdp_antiCausalCoeff, c.stdp_multiplier, c.stdp_tau_ms = anti, mult, tau
    c.stdp_causalMax, c.stdp_antiCausalMax = cmax, amax
    c.stdp_tauDecay_s, c.stdp_drift = tdec, drift
    c.delay_exp = 1 if getattr(cfg, "delay_exponential", False) else 0
    return c


def outdegree_by_delay(cfg, libm_mode: int = 0) -> np.ndarray:
    """(glob_n, D) uint16: synapses of each presynaptic neuron per delay slot,
    from the restatement's generation alone (any network size)."""
    c = config_from_netconfig(cfg)
    out = np.zeros((cfg.glob_n, cfg.D), np.uint16)
    if lib().dpo_outdegree_by_delay(C.byref(c), libm_mode, _ptr(out)) != 0:
        raise RuntimeError("oracle: " + lib().dpo_last_error().decode())
    return out


def events_per_step(outdeg: np.ndarray, ids: np.ndarray, ts: np.ndarray, total_ms: int) -> np.ndarray:
    """Synaptic events delivered at each step 0..total_ms-1 by the spikes of a
    raster: a spike emitted during ms m is compacted at step m+1 and its
    synapses of delay slot d are delivered at step m+1+d
    (DPSNN_localNet_sim.c:837-999)."""
    D = outdeg.shape[1]
    ev = np.zeros(total_ms + D + 1, np.int64)
    step0 = np.floor(ts).astype(np.int64) + 1
    for d in range(D):
        np.add.at(ev, step0 + d, outdeg[ids, d].astype(np.int64))
    return ev[:total_ms]


class OracleNet:
    """One network simulated by the CPU restatement."""

    def __init__(self, cfg, libm_mode: int = 0):
        self._L = lib()
        self._cfgs = config_from_netconfig(cfg)
        h = self._L.dpo_create(C.byref(self._cfgs), libm_mode)
        if not h:
            raise RuntimeError("oracle: " + self._L.dpo_last_error().decode())
        self._h = h
        self.glob_n = self._L.dpo_glob_n(h)
        self.loc_n = self._L.dpo_loc_n(h)
        self.glob_h = cfg.glob_h

    def close(self):
        if self._h:
            self._L.dpo_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synapses(self, rank: int = 0):
        n = self._L.dpo_rank_synapse_count(self._h, rank)
        pre = np.empty(n, np.uint32)
        post = np.empty(n, np.uint32)
        d = np.empty(n, np.uint8)
        k = np.empty(n, np.uint8)
        w = np.empty(n, np.int16)
        self._L.dpo_rank_synapses(self._h, rank, _ptr(pre), _ptr(post), _ptr(d), _ptr(k), _ptr(w))
        return pre, post, d, k, w

    def plasticity(self, rank: int = 0):
        n = self._L.dpo_rank_synapse_count(self._h, rank)
        td = np.empty(n, np.float32)
        la = np.empty(n, np.int32)
        self._L.dpo_rank_plasticity(self._h, rank, _ptr(td), _ptr(la))
        return td, la

    def bath_params(self):
        inv = np.empty(self.glob_n, np.float64)
        mx = np.empty(self.glob_n, np.uint32)
        self._L.dpo_bath_params(self._h, _ptr(inv), _ptr(mx))
        return inv, mx

    def lut(self, s: int):
        out = np.empty(256, np.float64)
        self._L.dpo_bath_lut(self._h, s, _ptr(out))
        return out

    def write_backward_dump(self, path: str):
        if self._L.dpo_write_backward_dump(self._h, path.encode()) != 0:
            raise OSError(path)

    def step(self):
        k = self._L.dpo_step(self._h)
        if k < 0:
            raise RuntimeError("oracle: " + self._L.dpo_last_error().decode())
        ids = np.empty(k, np.uint32)
        ts = np.empty(k, np.float64)
        if k:
            self._L.dpo_last_spikes(self._h, _ptr(ids), _ptr(ts))
        return ids, ts

    @property
    def time_ms(self):
        return self._L.dpo_time_ms(self._h)

    def last_event_count(self):
        return self._L.dpo_last_event_count(self._h)

    def last_bath_count(self):
        return self._L.dpo_last_bath_count(self._h)

    def state(self):
        arrs = [np.empty(self.glob_n, np.float64) for _ in range(5)]
        self._L.dpo_state(self._h, *[_ptr(a) for a in arrs])
        return dict(zip(("v", "c", "tr", "te", "nb"), arrs))


def ran3_sequence(seed: int, n: int) -> np.ndarray:
    out = np.empty(n, np.float64)
    lib().dpo_ran3_sequence(seed, n, _ptr(out))
    return out


def normdev_sequence(seed: int, n: int) -> np.ndarray:
    out = np.empty(n, np.float64)
    lib().dpo_normdev_sequence(seed, n, _ptr(out))
    return out


def gaussian_lut(mu, sigma, xmin, xmax) -> np.ndarray:
    out = np.empty(256, np.float64)
    lib().dpo_gaussian_lut(mu, sigma, xmin, xmax, _ptr(out))
    return out
