"""ctypes binding of the engine's C ABI (include/dpsnn_b200.h).

The engine library ``libdpsnn_b200.so`` is built in-tree by ``build()``
(csrc/Makefile).  There is no fallback: if the library or a GPU is missing,
constructing an :class:`Engine` raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdpsnn_b200.so")
MAX_SUB = 27


class Params(C.Structure):
    _fields_ = [
        ("cfx", C.c_uint32), ("cfy", C.c_uint32), ("nsub", C.c_uint32),
        ("count", C.c_uint32 * MAX_SUB),
        ("JExt", C.c_float * MAX_SUB), ("DJExt", C.c_float * MAX_SUB), ("NuExt", C.c_float * MAX_SUB),
        ("Tau", C.c_float * MAX_SUB), ("Theta", C.c_float * MAX_SUB), ("H", C.c_float * MAX_SUB),
        ("Tarp", C.c_float * MAX_SUB), ("AlphaC", C.c_float * MAX_SUB), ("TauC", C.c_float * MAX_SUB),
        ("gC", C.c_float * MAX_SUB),
        ("J", C.c_float * (MAX_SUB * MAX_SUB)), ("DJ", C.c_float * (MAX_SUB * MAX_SUB)),
        ("DMin", C.c_float * (MAX_SUB * MAX_SUB)), ("DMax", C.c_float * (MAX_SUB * MAX_SUB)),
        ("stencil_dim", C.c_uint32),
        ("spec", C.POINTER(C.c_float)),
        ("bath", C.POINTER(C.c_uint32)),
        ("D", C.c_uint32), ("glob_h", C.c_uint32), ("global_seed", C.c_uint32),
        ("total_sim_time_ms", C.c_uint32),
        ("start_plasticity_ms", C.c_uint32), ("stop_plasticity_ms", C.c_uint32),
        ("min_syn_weight_f", C.c_float),
        ("stdp_antiCausalCoeff", C.c_float), ("stdp_multiplier", C.c_float), ("stdp_tau_ms", C.c_float),
        ("stdp_causalMax", C.c_float), ("stdp_antiCausalMax", C.c_float), ("stdp_tauDecay_s", C.c_float),
        ("stdp_drift", C.c_float),
        ("moduloSec", C.c_uint32), ("ratesSampling", C.c_uint32),
        ("startStatFiles_s", C.c_uint32), ("stopStatFiles_s", C.c_uint32),
        ("startRatesPerPop_s", C.c_uint32), ("stopRatesPerPop_s", C.c_uint32),
        ("spikes_writeDisable", C.c_uint32), ("statRatesPerPop_writeDisable", C.c_uint32),
        ("howManyOutputFiles", C.c_uint32),
        ("delay_exponential", C.c_uint32),
    ]


class Options(C.Structure):
    _fields_ = [("events_per_neuron", C.c_uint32), ("overflow_events", C.c_uint32), ("device", C.c_int)]


EXPORTS = [
    "dpsnn_params_from_env", "dpsnn_create", "dpsnn_destroy", "dpsnn_step", "dpsnn_sync",
    "dpsnn_glob_n", "dpsnn_time_ms", "dpsnn_synapse_count", "dpsnn_events_delivered",
    "dpsnn_spikes", "dpsnn_rank_synapse_count", "dpsnn_backward_synapses", "dpsnn_state",
    "dpsnn_bath_params", "dpsnn_set_timing", "dpsnn_kernel_times", "dpsnn_kernel_launches", "dpsnn_cuda_stream",
    "dpsnn_rank_spikes_noalloc", "dpsnn_enable_ltp_probe", "dpsnn_ltp_probe",
    "dpsnn_enable_stdp_events", "dpsnn_stdp_events", "dpsnn_step_many", "dpsnn_last_error",
    "dpsnn_spikes_range", "dpsnn_device_bytes", "dpsnn_graph_create", "dpsnn_graph_run", "dpsnn_graph_destroy",
    "dpsnn_set_launch_shape",
]
NOALLOC_MAX_SPIKES = 32768   # DPSNN_NOALLOC_MAX_SPIKES
TIMING_SLOTS = 8             # DPSNN_TIMING_SLOTS
STDP_LOG_CAP = 1 << 21       # DPSNN_STDP_LOG_CAP
TIMING_NAMES = ["compact", "deliver", "bath", "neuron", "plasticity", "heavy_sort", "heavy_run", "huge"]

_LIB = None


def load_library(path: str = LIB_PATH):
    """Load the engine library (raises OSError when it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise OSError(f"{path} is missing: run __graft_entry__.build() first")
    lib = C.CDLL(path)
    P = C.c_void_p
    lib.dpsnn_params_from_env.argtypes = [C.c_char_p, C.POINTER(Params)]
    lib.dpsnn_create.argtypes = [C.POINTER(Params), C.POINTER(Options), C.POINTER(P)]
    lib.dpsnn_destroy.argtypes = [P]
    lib.dpsnn_destroy.restype = None
    lib.dpsnn_step.argtypes = [P, C.c_uint32]
    lib.dpsnn_sync.argtypes = [P]
    lib.dpsnn_glob_n.argtypes = [P]
    lib.dpsnn_glob_n.restype = C.c_uint32
    lib.dpsnn_time_ms.argtypes = [P]
    lib.dpsnn_time_ms.restype = C.c_uint32
    lib.dpsnn_synapse_count.argtypes = [P]
    lib.dpsnn_synapse_count.restype = C.c_uint64
    lib.dpsnn_events_delivered.argtypes = [P]
    lib.dpsnn_events_delivered.restype = C.c_uint64
    lib.dpsnn_spikes.argtypes = [P, C.c_uint32, P, P, C.c_uint32, C.POINTER(C.c_uint32)]
    lib.dpsnn_rank_synapse_count.argtypes = [P, C.c_uint32]
    lib.dpsnn_rank_synapse_count.restype = C.c_uint64
    lib.dpsnn_backward_synapses.argtypes = [P, C.c_uint32] + [P] * 6
    lib.dpsnn_state.argtypes = [P] * 6
    lib.dpsnn_bath_params.argtypes = [P, P, P]
    lib.dpsnn_set_timing.argtypes = [P, C.c_int]
    lib.dpsnn_kernel_times.argtypes = [P, P, P]
    lib.dpsnn_kernel_launches.argtypes = [P]
    lib.dpsnn_kernel_launches.restype = C.c_uint64
    lib.dpsnn_cuda_stream.argtypes = [P]
    lib.dpsnn_cuda_stream.restype = C.c_void_p
    lib.dpsnn_rank_spikes_noalloc.argtypes = [P, C.c_uint32, C.c_uint32, P, P, C.c_uint32,
                                              C.POINTER(C.c_uint32)]
    lib.dpsnn_enable_ltp_probe.argtypes = [P]
    lib.dpsnn_ltp_probe.argtypes = [P, C.c_uint32, C.POINTER(C.c_uint32)] + [P] * 4
    lib.dpsnn_enable_stdp_events.argtypes = [P]
    lib.dpsnn_stdp_events.argtypes = [P, C.POINTER(C.c_uint32), P, P, P, C.c_uint32, C.POINTER(C.c_uint32)]
    lib.dpsnn_step_many.argtypes = [P, C.c_uint32, C.c_uint32]
    lib.dpsnn_spikes_range.argtypes = [P, C.c_uint32, C.c_uint32, P, P, C.c_uint64, P]
    lib.dpsnn_device_bytes.argtypes = [P]
    lib.dpsnn_device_bytes.restype = C.c_uint64
    lib.dpsnn_graph_create.argtypes = [P, C.c_uint32, C.c_uint32, C.POINTER(P)]
    lib.dpsnn_graph_run.argtypes = [P]
    lib.dpsnn_graph_destroy.argtypes = [P]
    lib.dpsnn_graph_destroy.restype = None
    lib.dpsnn_set_launch_shape.argtypes = [P, C.c_uint32, C.c_uint32, C.c_uint32]
    lib.dpsnn_last_error.restype = C.c_char_p
    _LIB = lib
    return lib


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class ParamsHolder:
    """A Params struct together with the arrays its pointers refer to."""

    def __init__(self, p: Params, spec: np.ndarray, bath: np.ndarray):
        self.p, self.spec, self.bath = p, spec, bath


def params_from_netconfig(cfg) -> ParamsHolder:
    """Fill the engine's parameter struct from a ``netconfig.NetConfig``
    (the values the reference would read from the files it writes)."""
    p = Params()
    nsub = len(cfg.subpops)
    p.cfx, p.cfy, p.nsub = cfg.cfx, cfg.cfy, nsub
    f32 = lambda v: float(np.float32(v))
    for i, sp in enumerate(cfg.subpops):
        p.count[i] = sp.count
        for f in ("JExt", "DJExt", "NuExt", "Tau", "Theta", "H", "Tarp", "AlphaC", "TauC", "gC"):
            getattr(p, f)[i] = f32(getattr(sp, f))
    S = cfg.stencil_dim
    spec = np.zeros((nsub, nsub, S, S), np.float32)
    for (s, t), (J, DJ, dmin, dmax, probs) in cfg.conn.items():
        p.J[s * nsub + t], p.DJ[s * nsub + t] = f32(J), f32(DJ)
        p.DMin[s * nsub + t], p.DMax[s * nsub + t] = f32(dmin), f32(dmax)
        for y in range(S):
            for x in range(S):
                spec[s, t, x, y] = probs[y * S + x]
    bath = np.full((S, S), cfg.bath_cext, np.uint32)
    spec = np.ascontiguousarray(spec)
    p.stencil_dim = S
    p.spec = spec.ctypes.data_as(C.POINTER(C.c_float))
    p.bath = bath.ctypes.data_as(C.POINTER(C.c_uint32))
    p.D, p.glob_h, p.global_seed = cfg.D, cfg.glob_h, cfg.seed
    p.total_sim_time_ms = cfg.total_ms
    p.start_plasticity_ms, p.stop_plasticity_ms = cfg.start_plasticity_ms, cfg.stop_plasticity_ms
    p.min_syn_weight_f = f32(cfg.min_syn_weight_f)
    if cfg.stdp is not None:
        _, anti, mult, tau, cmax, amax, tdec, drift = cfg.stdp
    else:
        anti, mult, tau, cmax, amax, tdec, drift = -1.0, 0.001, 20.0, 0.1, 0.12, 1.0, 0.0
    p.stdp_antiCausalCoeff, p.stdp_multiplier, p.stdp_tau_ms = f32(anti), f32(mult), f32(tau)
    p.stdp_causalMax, p.stdp_antiCausalMax = f32(cmax), f32(amax)
    p.stdp_tauDecay_s, p.stdp_drift = f32(tdec), f32(drift)
    p.moduloSec, p.ratesSampling = 1, 5
    p.startStatFiles_s, p.stopStatFiles_s = 0, 100000
    p.startRatesPerPop_s, p.stopRatesPerPop_s = 0, 100000
    p.howManyOutputFiles = 1
    p.delay_exponential = 1 if getattr(cfg, "delay_exponential", False) else 0
    return ParamsHolder(p, spec, bath)


class EngineError(RuntimeError):
    pass


class Engine:
    """One network on one GPU."""

    def __init__(self, params, events_per_neuron: int = 0, overflow_events: int = 0, device: int = -1):
        self._L = load_library()
        holder = params if isinstance(params, ParamsHolder) else params_from_netconfig(params)
        self._holder = holder
        opts = Options(events_per_neuron, overflow_events, device)
        h = C.c_void_p()
        rc = self._L.dpsnn_create(C.byref(holder.p), C.byref(opts), C.byref(h))
        if rc != 0:
            raise EngineError(f"dpsnn_create failed ({rc}): {self._L.dpsnn_last_error().decode()}")
        self._h = h
        self.glob_n = self._L.dpsnn_glob_n(h)
        self.glob_h = holder.p.glob_h

    def _check(self, rc, what):
        if rc != 0:
            raise EngineError(f"{what} failed ({rc}): {self._L.dpsnn_last_error().decode()}")

    def close(self):
        if getattr(self, "_h", None):
            self._L.dpsnn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n: int = 1):
        self._check(self._L.dpsnn_step(self._h, n), "dpsnn_step")

    def sync(self):
        self._check(self._L.dpsnn_sync(self._h), "dpsnn_sync")

    @property
    def time_ms(self) -> int:
        return self._L.dpsnn_time_ms(self._h)

    @property
    def synapse_count(self) -> int:
        return self._L.dpsnn_synapse_count(self._h)

    def events_delivered(self) -> int:
        return self._L.dpsnn_events_delivered(self._h)

    def spikes(self, t_ms: int):
        """(ids, emission times) of the spikes detected at step t_ms."""
        if getattr(self, "_sbuf", None) is None:
            self._sbuf = (np.empty(self.glob_n, np.uint32), np.empty(self.glob_n, np.float64))
        ids, te = self._sbuf
        cnt = C.c_uint32()
        self._check(self._L.dpsnn_spikes(self._h, t_ms, _ptr(ids), _ptr(te), self.glob_n, C.byref(cnt)),
                    "dpsnn_spikes")
        n = cnt.value
        return ids[:n].copy(), te[:n].copy()

    def spikes_range(self, t0: int, n: int):
        """(ids, emission times, per-step counts) of the spikes detected at
        steps t0 .. t0+n-1, concatenated in step order (one wait)."""
        cap = max(self.glob_n * n, 1)
        if getattr(self, "_rbuf", None) is None or len(self._rbuf[0]) < cap:
            self._rbuf = (np.empty(cap, np.uint32), np.empty(cap, np.float64))
        ids, te = self._rbuf
        counts = np.zeros(max(n, 1), np.uint32)
        self._check(self._L.dpsnn_spikes_range(self._h, t0, n, _ptr(ids), _ptr(te), cap, _ptr(counts)),
                    "dpsnn_spikes_range")
        k = int(counts[:n].sum())
        return ids[:k].copy(), te[:k].copy(), counts[:n]

    @property
    def device_bytes(self) -> int:
        """Device memory the engine holds."""
        return self._L.dpsnn_device_bytes(self._h)

    def set_launch_shape(self, deliver_blocks: int = 0, heavy_sort_blocks: int = 0, heavy_run_blocks: int = 0):
        """Grid sizes of the delivery, warp-sort and heavy-run kernels (0 =
        the defaults, sized for a network that fills the GPU); results do
        not depend on them."""
        self._check(self._L.dpsnn_set_launch_shape(self._h, deliver_blocks, heavy_sort_blocks, heavy_run_blocks),
                    "dpsnn_set_launch_shape")

    def rank_spikes_noalloc(self, t_ms: int, rank: int):
        """Spikes of one emulated rank at step t_ms, gathered without any
        device allocation (dpsnn_rank_spikes_noalloc)."""
        cnt = C.c_uint32()
        cap = NOALLOC_MAX_SPIKES
        ids = np.empty(cap, np.uint32)
        te = np.empty(cap, np.float64)
        self._check(self._L.dpsnn_rank_spikes_noalloc(self._h, t_ms, rank, _ptr(ids), _ptr(te), cap,
                                                        C.byref(cnt)), "dpsnn_rank_spikes_noalloc")
        n = cnt.value
        return ids[:n].copy(), te[:n].copy()

    def backward_synapses(self, rank: int = 0, with_tderiv: bool = False):
        n = self._L.dpsnn_rank_synapse_count(self._h, rank)
        pre = np.empty(n, np.uint32)
        post = np.empty(n, np.uint32)
        d = np.empty(n, np.uint8)
        k = np.empty(n, np.uint8)
        w = np.empty(n, np.int16)
        td = np.empty(n, np.float32) if with_tderiv else None
        self._check(self._L.dpsnn_backward_synapses(self._h, rank, _ptr(pre), _ptr(post), _ptr(d), _ptr(k),
                                                     _ptr(w), _ptr(td)), "dpsnn_backward_synapses")
        return (pre, post, d, k, w, td) if with_tderiv else (pre, post, d, k, w)

    def enable_ltp_probe(self):
        """Keep the synapses around each plasticity update (before the first step)."""
        self._check(self._L.dpsnn_enable_ltp_probe(self._h), "dpsnn_enable_ltp_probe")

    def ltp_probe(self, rank: int = 0):
        """(step, w_before, td_before, w_after, td_after) of the last plasticity
        update, in the order of :meth:`backward_synapses`."""
        n = self._L.dpsnn_rank_synapse_count(self._h, rank)
        wb, wa = np.empty(n, np.int16), np.empty(n, np.int16)
        tb, ta = np.empty(n, np.float32), np.empty(n, np.float32)
        t = C.c_uint32(0)
        self._check(self._L.dpsnn_ltp_probe(self._h, rank, C.byref(t), _ptr(wb), _ptr(tb), _ptr(wa), _ptr(ta)),
                    "dpsnn_ltp_probe")
        return t.value, wb, tb, wa, ta

    def enable_stdp_events(self):
        """Log every step's rank-0 STDP contributions (before the first step)."""
        self._check(self._L.dpsnn_enable_stdp_events(self._h), "dpsnn_enable_stdp_events")

    def stdp_events(self):
        """(step, pre, post, contribution) of the last step queued, in the
        reference's order."""
        cap = STDP_LOG_CAP
        pre, post = np.empty(cap, np.uint32), np.empty(cap, np.uint32)
        c = np.empty(cap, np.float32)
        t, n = C.c_uint32(0), C.c_uint32(0)
        self._check(self._L.dpsnn_stdp_events(self._h, C.byref(t), _ptr(pre), _ptr(post), _ptr(c), cap,
                                              C.byref(n)), "dpsnn_stdp_events")
        return t.value, pre[:n.value].copy(), post[:n.value].copy(), c[:n.value].copy()

    def state(self):
        arrs = [np.empty(self.glob_n, np.float64) for _ in range(5)]
        self._check(self._L.dpsnn_state(self._h, *[_ptr(a) for a in arrs]), "dpsnn_state")
        return dict(zip(("v", "c", "tr", "te", "nb"), arrs))

    def bath_params(self):
        inv = np.empty(self.glob_n, np.float64)
        mx = np.empty(self.glob_n, np.uint32)
        self._check(self._L.dpsnn_bath_params(self._h, _ptr(inv), _ptr(mx)), "dpsnn_bath_params")
        return inv, mx

    def set_timing(self, on: bool):
        self._check(self._L.dpsnn_set_timing(self._h, 1 if on else 0), "dpsnn_set_timing")

    def cuda_stream(self) -> int:
        return self._L.dpsnn_cuda_stream(self._h)

    def kernel_launches(self) -> int:
        return self._L.dpsnn_kernel_launches(self._h)

    def kernel_times(self):
        sec = np.zeros(TIMING_SLOTS, np.float64)
        cnt = np.zeros(TIMING_SLOTS, np.uint64)
        self._check(self._L.dpsnn_kernel_times(self._h, _ptr(sec), _ptr(cnt)), "dpsnn_kernel_times")
        return sec, cnt


def params_from_env(workdir: str) -> ParamsHolder:
    """Parse env_* + input files in ``workdir`` with the engine's C parser."""
    lib = load_library()
    p = Params()
    rc = lib.dpsnn_params_from_env(workdir.encode(), C.byref(p))
    if rc != 0:
        raise EngineError(f"dpsnn_params_from_env failed ({rc}): {lib.dpsnn_last_error().decode()}")
    nsub, S = p.nsub, p.stencil_dim
    spec = np.ctypeslib.as_array(p.spec, shape=(nsub * nsub * S * S,)).copy()
    bath = np.ctypeslib.as_array(p.bath, shape=(S * S,)).copy()
    p.spec = spec.ctypes.data_as(C.POINTER(C.c_float))
    p.bath = bath.ctypes.data_as(C.POINTER(C.c_uint32))
    return ParamsHolder(p, spec, bath)


def step_many(engines, n: int):
    """The batched form: ``n`` steps of each engine, queued one step of every
    engine at a time so that independent networks overlap on the device."""
    lib = load_library()
    arr = (C.c_void_p * len(engines))(*[e._h for e in engines])
    rc = lib.dpsnn_step_many(arr, len(engines), n)
    if rc != 0:
        raise EngineError(f"dpsnn_step_many failed ({rc}): {lib.dpsnn_last_error().decode()}")


class Graph:
    """``nsteps`` steps (a multiple of 80) of every engine, in
    :func:`step_many`'s order, recorded once into a CUDA graph
    (dpsnn_graph_create); :meth:`run` advances every engine by ``nsteps``
    steps in one launch.  The engines must have run their first step."""

    def __init__(self, engines, nsteps: int):
        self._L = load_library()
        self.engines = list(engines)
        self.nsteps = nsteps
        arr = (C.c_void_p * len(self.engines))(*[e._h for e in self.engines])
        g = C.c_void_p()
        rc = self._L.dpsnn_graph_create(arr, len(self.engines), nsteps, C.byref(g))
        if rc != 0:
            raise EngineError(f"dpsnn_graph_create failed ({rc}): {self._L.dpsnn_last_error().decode()}")
        self._g = g

    def run(self):
        rc = self._L.dpsnn_graph_run(self._g)
        if rc != 0:
            raise EngineError(f"dpsnn_graph_run failed ({rc}): {self._L.dpsnn_last_error().decode()}")

    def close(self):
        if self._g:
            self._L.dpsnn_graph_destroy(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
