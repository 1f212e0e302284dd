"""Input files and environment for one DPSNN run.

The reference reads its network from four text files in the working
directory and about thirty ``env_*`` variables:

* ``column.txt``      -- one row per sub-population:
  ``subPop count JExt DJExt NuExt Tau Theta H Tarp AlphaC TauC gC``
  (parsed by ``initSubPopParamStruct``, DPSNN_LIFCAconnectome.cpp:302-398,
  and counted by ``readColumnFile``, DPSNN_getParameters.c:834-898);
* ``connectivity.txt`` -- one row per (source, target) sub-population pair:
  ``src tgt J DJ DMin DMax p[x][y] ...`` with the stencil probabilities in
  y-major order (``initConnectivityParam``, DPSNN_LIFCAconnectome.cpp:16-131);
* ``bathEfficacy.txt`` -- ``stencilDim`` rows of ``stencilDim`` integers,
  the external-bath in-degree CExt (DPSNN_LIFCAconnectome.cpp:240-300);
* ``plasticity.txt``  -- one line ``1 antiCausalCoeff STDPmultiplier tauSTDP
  causalMax antiCausalMax tauDerivativeDecay_s derivativeDrift``
  (``readPlasticityParametersFile``, DPSNN_getParameters.c:900-1053; the
  reference keeps the *last* line it reads, so the parameter line is last).

The reference ships none of these files.  :func:`cortical_grid` authors them
for the benchmark family: modules of 500+500 excitatory LIFCA neurons and 250
inhibitory LIF neurons, intra-module connection probability 0.8, lateral
probability ``p1 * exp(-(d - 1))`` at Euclidean module distance ``d`` inside
a ``(2*stencil-1)^2`` stencil, uniform integer delays of 1-20 ms, Gaussian
weights N(mu, 0.1 mu) (excitatory) and N(-4 mu, 0.4 mu) (inhibitory), and a
3 kHz Poisson bath of efficacy N(mu, 0.1 mu).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional

__all__ = ["SubPop", "NetConfig", "cortical_grid", "lateral_p1_for_grid"]


@dataclass
class SubPop:
    count: int
    JExt: float
    DJExt: float
    NuExt: float
    Tau: float
    Theta: float
    H: float
    Tarp: float
    AlphaC: float
    TauC: float
    gC: float


@dataclass
class NetConfig:
    """Everything one reference run reads: files plus environment."""

    cfx: int
    cfy: int
    subpops: List[SubPop]
    # conn[(src, tgt)] = (J, DJ, DMin, DMax, [p[x][y] in y-major order])
    conn: Dict[tuple, tuple]
    stencil_dim: int
    bath_cext: int = 1000
    total_ms: int = 1000
    glob_h: int = 1
    seed: int = 1
    D: int = 21
    min_syn_weight_f: float = -6.0
    stdp: Optional[tuple] = None          # plasticity.txt row, or None
    start_plasticity_ms: int = 10 ** 8
    stop_plasticity_ms: int = 10 ** 8
    # getRandomDelay_EXP instead of getRandomDelay_UNI: the reference picks it
    # at compile time (no -DDelayUniform); the engine reads DPSNN_DELAY_DISTRIBUTION
    delay_exponential: bool = False
    extra_env: Dict[str, str] = field(default_factory=dict)

    @property
    def neurons_per_module(self) -> int:
        return sum(p.count for p in self.subpops)

    @property
    def n_modules(self) -> int:
        return self.cfx * self.cfy

    @property
    def glob_n(self) -> int:
        return self.neurons_per_module * self.n_modules

    # -- files ---------------------------------------------------------
    def column_txt(self) -> str:
        rows = []
        for i, p in enumerate(self.subpops):
            rows.append(" ".join(_fmt(v) for v in (
                i, p.count, p.JExt, p.DJExt, p.NuExt, p.Tau, p.Theta, p.H,
                p.Tarp, p.AlphaC, p.TauC, p.gC)))
        # no blank lines: readColumnFile dereferences the token of every line
        return "\n".join(rows) + "\n"

    def connectivity_txt(self) -> str:
        rows = []
        for (s, t), (J, DJ, dmin, dmax, probs) in sorted(self.conn.items()):
            rows.append(" ".join(_fmt(v) for v in (s, t, J, DJ, dmin, dmax, *probs)))
        return "\n".join(rows) + "\n"

    def bath_efficacy_txt(self) -> str:
        row = " ".join(str(self.bath_cext) for _ in range(self.stencil_dim))
        return "\n".join(row for _ in range(self.stencil_dim)) + "\n"

    def plasticity_txt(self) -> Optional[str]:
        if self.stdp is None:
            return None
        return " ".join(_fmt(v) for v in self.stdp) + "\n"

    def env(self) -> Dict[str, str]:
        e = {
            "env_overallConnectivity": "0",
            "env_stencilDim": str(self.stencil_dim),
            "env_synGen": "2",
            "env_globH": str(self.glob_h),
            "env_CFX": str(self.cfx),
            "env_CFY": str(self.cfy),
            "env_D": str(self.D),
            "env_chrono": "1",
            "env_startPartialChrono_ms": "0",
            "env_partialChronoWindow_ms": str(self.total_ms),
            "env_totalSimTime_ms": str(self.total_ms),
            "env_startPlasticity_ms": str(self.start_plasticity_ms),
            "env_stopPlasticity_ms": str(self.stop_plasticity_ms),
            "env_moduloSec": "1",
            "env_startStatFiles_s": "0",
            "env_stopStatFiles_s": "100000",
            "env_spikes_writeDisable": "0",
            "env_statSTDPevent_writeDisable": "1",
            "env_statSynPeriodicProbe_writeDisable": "1",
            "env_statRatesPerPop_writeDisable": "0",
            "env_startRatesPerPop_s": "0",
            "env_stopRatesPerPop_s": "100000",
            "env_startSynPeriodicProbe_s": "0",
            "env_stopSynPeriodicProbe_s": "0",
            "env_startSTDPevent_s": "0",
            "env_stopSTDPevent_s": "0",
            "env_ratesSampling": "5",
            "env_fastDebugDyn": "0",
            "env_debugPrintEnable_ms": "0",
            "env_globalSeed": str(self.seed),
            "env_howManyOutputFiles": "1",
            "env_minSynWeight_f": _fmt(self.min_syn_weight_f),
            "env_collectivesAlgo": "0",
            "env_pktLength": "0",
        }
        if self.delay_exponential:
            e["DPSNN_DELAY_DISTRIBUTION"] = "exponential"
        e.update(self.extra_env)
        return e

    def write(self, directory: str) -> Dict[str, str]:
        """Write the input files into ``directory``; return the environment."""
        os.makedirs(directory, exist_ok=True)
        files = {
            "column.txt": self.column_txt(),
            "connectivity.txt": self.connectivity_txt(),
            "bathEfficacy.txt": self.bath_efficacy_txt(),
        }
        pl = self.plasticity_txt()
        if pl is not None:
            files["plasticity.txt"] = pl
        else:
            stale = os.path.join(directory, "plasticity.txt")
            if os.path.exists(stale):
                os.remove(stale)
        for name, text in files.items():
            with open(os.path.join(directory, name), "w") as f:
                f.write(text)
        return self.env()


def _fmt(v) -> str:
    if isinstance(v, int):
        return str(v)
    return repr(float(v))


def _stencil_probs(stencil_dim: int, p_intra: float, p1: float, lam: float) -> List[float]:
    """Probabilities p[x][y], x,y in 0..stencil_dim-1, listed y-major."""
    out = []
    for y in range(stencil_dim):
        for x in range(stencil_dim):
            if x == 0 and y == 0:
                out.append(p_intra)
            else:
                d = math.hypot(x, y)
                out.append(p1 * math.exp(-(d - 1.0) / lam))
    return out


def lateral_p1_for_grid(cfx: int, cfy: int, stencil_dim: int = 2, lam: float = 1.0,
                        neurons_per_module: int = 1250,
                        lateral_indegree: float = 125.0) -> float:
    """p1 such that the grid-mean lateral in-degree is ``lateral_indegree``."""
    tot = 0.0
    for ty in range(cfy):
        for tx in range(cfx):
            for dy in range(-(stencil_dim - 1), stencil_dim):
                for dx in range(-(stencil_dim - 1), stencil_dim):
                    if dx == 0 and dy == 0:
                        continue
                    sx, sy = tx + dx, ty + dy
                    if 0 <= sx < cfx and 0 <= sy < cfy:
                        tot += math.exp(-(math.hypot(dx, dy) - 1.0) / lam)
    mean_weight = tot / (cfx * cfy)
    if mean_weight == 0:   # a single module: no lateral connections at all
        return 0.0
    return lateral_indegree / (neurons_per_module * mean_weight)


def cortical_grid(cfx: int, cfy: int, *, mu: float = 0.3, g_c: float = 3.0,
                  alpha_c: float = 1.0, nu_ext_hz: float = 3.0,
                  n_exc_a: int = 500, n_exc_b: int = 500, n_inh: int = 250,
                  stencil_dim: int = 2, p_intra: float = 0.8,
                  p1: Optional[float] = None, lam: float = 1.0,
                  total_ms: int = 1000, seed: int = 1, glob_h: int = 1,
                  stdp: bool = False, start_plasticity_ms: int = 0,
                  delay_exponential: bool = False, delay_range_subpop: bool = False) -> NetConfig:
    """The benchmark network family (see module docstring).

    ``delay_range_subpop`` adds a fourth, empty sub-population (0 neurons, no
    connection in or out) whose self-pair row declares DMax = 21 ms.  The
    reference keeps the delay range of the whole problem as integers
    (``delayMin``/``delayMax`` are uint32_t, DPSNN_parameters.h:111-112, set at
    DPSNN_LIFCAconnectome.cpp:467-480) and splits it into 80 levels; with the
    range 1-20 ms, getRandomDelay_UNI (DPSNN_LIFCAcorticalModuleGen.cpp:299-338)
    maps the 60 largest of the 1e9 ran3 values to the float level 80.0 and
    stops the run ("delay level generated ... max allowed delay levels"), so
    the reference refuses any 1-20 ms network with more than a few tens of
    millions of synapses (6x6 modules and up).  With the range 1-21 ms the
    real pairs (DMin 1, DMax 20) use 76 levels of 0.25 ms: the same integer
    delays 1-20 ms with the same weights (half-weight endpoints), and the
    largest level is 76.0, so the reference builds every such network.
    """
    if p1 is None:
        # 0.0376 at 2x2 reproduces the ~1125 in-degree of the 2x2 benchmark;
        # larger grids use the value giving the same grid-mean in-degree.
        p1 = 0.0376 if (cfx, cfy) == (2, 2) and stencil_dim == 2 else \
            lateral_p1_for_grid(cfx, cfy, stencil_dim, lam, n_exc_a + n_exc_b + n_inh)
    exc = dict(JExt=mu, DJExt=0.1, NuExt=nu_ext_hz, Tau=20.0, Theta=20.0, H=15.0,
               Tarp=2.0, AlphaC=alpha_c, TauC=150.0, gC=g_c)
    inh = dict(JExt=mu, DJExt=0.1, NuExt=nu_ext_hz, Tau=10.0, Theta=20.0, H=15.0,
               Tarp=2.0, AlphaC=0.0, TauC=150.0, gC=0.0)
    subpops = [SubPop(n_exc_a, **exc), SubPop(n_exc_b, **exc), SubPop(n_inh, **inh)]
    probs = _stencil_probs(stencil_dim, p_intra, p1, lam)
    conn = {}
    for s in range(3):
        J = mu if s < 2 else -4.0 * mu
        for t in range(3):
            conn[(s, t)] = (J, 0.1, 1.0, 20.0, probs)
    if delay_range_subpop:
        subpops.append(SubPop(0, **exc))
        no_link = [0.0] * len(probs)
        for s in range(4):
            for t in range(4):
                if s == 3 or t == 3:
                    conn[(s, t)] = (mu, 0.1, 1.0, 21.0 if (s, t) == (3, 3) else 20.0, no_link)
    cfg = NetConfig(cfx=cfx, cfy=cfy, subpops=subpops, conn=conn,
                    stencil_dim=stencil_dim, total_ms=total_ms, seed=seed,
                    glob_h=glob_h, delay_exponential=delay_exponential)
    if stdp:
        cfg.stdp = (1, -1, 0.1, 20, 0.1, 0.12, 1, 0)
        cfg.start_plasticity_ms = start_plasticity_ms
        cfg.stop_plasticity_ms = 10 ** 8
    return cfg
