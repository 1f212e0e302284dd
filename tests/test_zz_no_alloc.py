"""dpsnn_rank_spikes_noalloc against dpsnn_spikes: the same rank's spike
list on two calls in a row, for every rank and for consecutive steps; ranks
larger than the fixed scratch are rejected; calls leave the device's free
memory unchanged.  Collected last (file name), and independent of the tests
before it."""
import numpy as np
import pytest

from tests.conftest import engine_module
from tests.golden.cases import CASES, small

pytestmark = pytest.mark.gpu
E = engine_module()


def rank_slice(ids, te, rank, loc_n):
    sel = (ids >= rank * loc_n) & (ids < (rank + 1) * loc_n)
    return ids[sel], te[sel]


def test_matches_spike_list_on_two_calls_in_a_row():
    cfg = CASES["small_2x2"]()
    cfg.glob_h = 4
    eng = E.Engine(cfg)
    loc_n = eng.glob_n // 4
    seen = 0
    for _ in range(12):
        eng.step(10)
        for t in (eng.time_ms - 2, eng.time_ms - 1):
            ids, te = eng.spikes(t)
            for h in range(4):
                want = rank_slice(ids, te, h, loc_n)
                for _call in range(2):
                    got = eng.rank_spikes_noalloc(t, h)
                    np.testing.assert_array_equal(got[0], want[0])
                    np.testing.assert_array_equal(got[1], want[1])
                seen += len(want[0])
    assert seen > 0
    eng.close()


def test_single_rank_and_empty_steps():
    cfg = CASES["small_1x1"]()
    eng = E.Engine(cfg)
    for t in range(30):
        eng.step(1)
        ids, te = eng.spikes(t)
        for _call in range(2):
            got = eng.rank_spikes_noalloc(t, 0)
            np.testing.assert_array_equal(got[0], ids)
            np.testing.assert_array_equal(got[1], te)
    with pytest.raises(E.EngineError, match="out of range"):
        eng.rank_spikes_noalloc(0, 1)
    eng.close()


def test_rejects_rank_larger_than_scratch():
    cfg = small(19, 19, ms=10)     # 36100 neurons on one rank > 32768
    eng = E.Engine(cfg)
    eng.step(1)
    with pytest.raises(E.EngineError, match="exceeds the 32768-spike scratch"):
        eng.rank_spikes_noalloc(0, 0)
    eng.close()


def test_device_memory_unchanged_over_many_calls():
    """No call allocates: the device's free memory is the same before and
    after 100 calls (after a first call, which looks up the scratch address,
    and with the engine's queued work finished)."""
    import torch
    cfg = CASES["small_2x2"]()
    cfg.glob_h = 4
    eng = E.Engine(cfg)
    eng.step(40)
    eng.sync()
    eng.rank_spikes_noalloc(39, 0)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for k in range(100):
        eng.rank_spikes_noalloc(39 - (k % 40), k % 4)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0
    eng.close()
