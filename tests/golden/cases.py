"""Networks pinned by the golden fixtures (see make_golden.py)."""
import importlib

nc = importlib.import_module("201812realtimecortsim_b200.netconfig")


def small(cfx, cfy, ms=300, mu=0.6, **kw):
    """Modules of 40+40 excitatory and 20 inhibitory neurons."""
    return nc.cortical_grid(cfx, cfy, n_exc_a=40, n_exc_b=40, n_inh=20, p1=0.2, total_ms=ms, mu=mu, **kw)


CASES = {
    # one module of 100 neurons
    "small_1x1": lambda: small(1, 1),
    # 2x2 modules of 100 neurons, seed 7
    "small_2x2": lambda: small(2, 2, seed=7),
    # same grid with Song STDP from t=0 through two weight updates (x999 ms)
    "small_2x2_stdp": lambda: small(2, 2, ms=2100, stdp=True, start_plasticity_ms=0),
    # the 2x2 benchmark network: 5000 neurons, ~5.6 M synapses, 1 s
    "c1_2x2": lambda: nc.cortical_grid(2, 2, total_ms=1000),
    # several MPI ranks (env_globH), run by the reference as that many
    # processes: each rank's own RNG streams, synapse lists and files
    "small_2x2_p4": lambda: small(2, 2, seed=7, glob_h=4),
    "small_2x2_stdp_p2": lambda: small(2, 2, ms=2100, stdp=True, start_plasticity_ms=0, glob_h=2),
    "c1_2x2_p4": lambda: nc.cortical_grid(2, 2, total_ms=1000, glob_h=4),
    # the reference Makefile's default delay distribution (getRandomDelay_EXP,
    # built without -DDelayUniform)
    "small_2x2_exp": lambda: small(2, 2, seed=7, delay_exponential=True),
    "c1_2x2_exp": lambda: nc.cortical_grid(2, 2, total_ms=1000, delay_exponential=True),
}


# Networks pinned by digests of the reference's raster (make_golden.py
# writes <name>.summary.npz): too large to commit the raster itself.  They
# use the delay-range sub-population (netconfig.cortical_grid), without which
# the reference refuses networks of 6x6 modules and more; the 2x2 network
# is the benchmark one, which the reference accepts as it is.  Per case: the network, the
# ranks whose BACKWARD synapse dump is hashed, and the window (ms) of the
# per-population firing statistics.  (The reference writes the dump of rank
# 0 only, DPSNN_localNet_init.c:786.)
SUMMARY_CASES = {
    # the benchmark network, 192 ranks (3 modules each), over its onset burst
    "c2_24x24_p192": (lambda: nc.cortical_grid(24, 24, total_ms=100, glob_h=192, delay_range_subpop=True),
                      (0,), (20, 100)),
    # 6x6 modules, 12 ranks, 10 s: the bit-identical window and, after it,
    # the firing statistics
    "c_6x6_p12_10s": (lambda: nc.cortical_grid(6, 6, total_ms=10000, glob_h=12, delay_range_subpop=True),
                      (0,), (1000, 10000)),
    # the 2x2 benchmark network, 1 rank, 10 s
    "c1_2x2_10s": (lambda: nc.cortical_grid(2, 2, total_ms=10000), (0,), (1000, 10000)),
    # the plasticity configuration on a 4x4 subgrid (20000 neurons, 1 rank):
    # pair-based additive STDP on E->E synapses (A+ 0.01, A- 0.012, tau 20 ms,
    # weights clipped to [0, 2 mu], updated each second) from t = 0, through
    # two weight updates (ms 999 and 1999)
    "c3_4x4_stdp": (lambda: nc.cortical_grid(4, 4, total_ms=2100, stdp=True, start_plasticity_ms=0,
                                             delay_range_subpop=True), (0,), (1000, 2100)),
}


# Networks the reference refuses to build; make_golden.py records its error
# line.  6x6 modules with delays 1-20 ms: one of the ~50 M delay draws
# reaches the float level 80 of getRandomDelay_UNI.
REFUSED_CASES = {
    "refused_6x6_p12": lambda: nc.cortical_grid(6, 6, total_ms=10, glob_h=12),
}
