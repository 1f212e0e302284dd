"""GPU engine parity: connectome, raster and state against the reference's
golden outputs and the CPU restatement, through the C ABI (ctypes)."""
import numpy as np
import pytest

import dpsnn_oracle as O
from tests.conftest import engine_module, netconfig
from tests.golden import io as gio
from tests.golden.cases import CASES, REFUSED_CASES, small

pytestmark = pytest.mark.gpu
E = engine_module()
nc = netconfig()


def run_engine(cfg, steps, chunk=50):
    eng = E.Engine(cfg)
    ids, ts = [], []
    done = 0
    while done < steps:
        k = min(chunk, steps - done)
        eng.step(k)
        for t in range(done, done + k):
            i, tt = eng.spikes(t)
            ids.append(i)
            ts.append(tt)
        done += k
    return eng, np.concatenate(ids), np.concatenate(ts)


@pytest.mark.parametrize("name", sorted(CASES))
def test_raster_identical_to_reference(name):
    cfg = CASES[name]()
    eng, ids, ts = run_engine(cfg, cfg.total_ms)
    ids, ts = gio.rank_major(ids, ts, cfg.glob_h, eng.glob_n)
    gi, gt = gio.raster(name)
    assert len(ids) == len(gi)
    np.testing.assert_array_equal(ids, gi)
    np.testing.assert_array_equal(ts, gt)


@pytest.mark.parametrize("name", ["small_1x1", "small_2x2", "c1_2x2", "c1_2x2_exp"])
def test_connectome_identical_to_oracle(name):
    cfg = CASES[name]()
    eng = E.Engine(cfg)
    orc = O.OracleNet(cfg)
    for g, o in zip(eng.backward_synapses(0), orc.synapses(0)):
        np.testing.assert_array_equal(g, o)
    gi, gm = eng.bath_params()
    oi, om = orc.bath_params()
    np.testing.assert_array_equal(gi, oi)
    np.testing.assert_array_equal(gm, om)


@pytest.mark.parametrize("ranks", [2, 4])
def test_emulated_ranks_match_oracle(ranks):
    # Several reference processes (env_globH > 1): per-rank RNG streams,
    # per-rank backward lists; checked against the restatement.
    cfg = small(2, 2, ms=400, seed=3, glob_h=ranks)
    eng, ids, ts = run_engine(cfg, cfg.total_ms)
    orc = O.OracleNet(cfg, 1)
    for h in range(ranks):
        for g, o in zip(eng.backward_synapses(h), orc.synapses(h)):
            np.testing.assert_array_equal(g, o)
    oi, ot = [], []
    for _ in range(cfg.total_ms):
        i, t = orc.step()
        oi.append(i)
        ot.append(t)
    np.testing.assert_array_equal(ids, np.concatenate(oi))
    np.testing.assert_array_equal(ts, np.concatenate(ot))
    st, so = eng.state(), orc.state()
    for k in st:
        np.testing.assert_array_equal(st[k], so[k])


def test_stdp_weights_and_traces_match_oracle():
    cfg = small(2, 2, ms=1100, seed=5, glob_h=2, stdp=True, start_plasticity_ms=0)
    eng, _, _ = run_engine(cfg, cfg.total_ms)
    orc = O.OracleNet(cfg, 1)
    for _ in range(cfg.total_ms):
        orc.step()
    for h in range(2):
        g = eng.backward_synapses(h, with_tderiv=True)
        o = orc.synapses(h)
        np.testing.assert_array_equal(g[4], o[4])          # int16 weights after x999
        np.testing.assert_array_equal(g[5], orc.plasticity(h)[0])


def test_run_to_run_determinism_large_grid():
    # 6x6 grid, 12 emulated ranks: atomics in delivery must not change results.
    cfg = nc.cortical_grid(6, 6, total_ms=60, glob_h=12, delay_range_subpop=True)
    a, ia, ta = run_engine(cfg, 60)
    b, ib, tb = run_engine(cfg, 60)
    np.testing.assert_array_equal(ia, ib)
    np.testing.assert_array_equal(ta, tb)
    sa, sb = a.state(), b.state()
    for k in sa:
        np.testing.assert_array_equal(sa[k], sb[k])


def test_full_size_grid_invariants():
    # 24x24 grid (720000 neurons, ~0.81 G synapses), 192 emulated ranks:
    # size-independent properties of the connectome and of the dynamics.
    cfg = nc.cortical_grid(24, 24, total_ms=40, glob_h=192, delay_range_subpop=True)
    eng = E.Engine(cfg)
    S = eng.synapse_count
    assert 0.79e9 < S < 0.83e9                   # mean in-degree ~1125
    eng.step(40)
    eng.sync()
    prev_hi = -1.0
    for t in range(40):
        ids, te = eng.spikes(t)
        assert np.all(np.diff(ids.astype(np.int64)) > 0)        # ascending index
        if len(te):
            assert te.min() >= t - 1 and te.max() < t             # emitted in step t-1
    assert eng.events_delivered() > 0


@pytest.mark.parametrize("name", sorted(REFUSED_CASES))
def test_refuses_what_the_reference_refuses(name):
    # e.g. 6x6 modules with delays 1-20 ms (no delay-range sub-population):
    # one of the ~50 M delay draws reaches level 80, where getRandomDelay_UNI
    # (DPSNN_LIFCAcorticalModuleGen.cpp:322-326) stops the reference with
    # "delay level generated ... max allowed delay levels"
    assert "delay level generated" in gio.manifest()[name]["refused"]
    with pytest.raises(E.EngineError, match="delay level generated"):
        E.Engine(REFUSED_CASES[name]())
