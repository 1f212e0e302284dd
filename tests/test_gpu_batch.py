"""The batched form (dpsnn_step_many): independent networks stepped together,
their kernels overlapping on the device, give each network exactly the raster
it gives alone, and the golden networks among them the reference's raster."""
import numpy as np
import pytest

from tests.conftest import engine_module
from tests.golden import io as gio
from tests.golden.cases import CASES, small

pytestmark = pytest.mark.gpu
E = engine_module()


def rasters_stepped_together(cfgs, steps, chunk=40):
    engines = [E.Engine(c) for c in cfgs]
    out = [([], []) for _ in cfgs]
    done = 0
    while done < steps:
        k = min(chunk, steps - done)   # spike lists stay readable for 80 steps
        E.step_many(engines, k)
        for e, (ids, ts) in zip(engines, out):
            for t in range(done, done + k):
                i, tt = e.spikes(t)
                ids.append(i)
                ts.append(tt)
        done += k
    res = [(np.concatenate(i), np.concatenate(t)) for i, t in out]
    ev = [e.events_delivered() for e in engines]
    for e in engines:
        e.close()
    return res, ev


def test_batched_networks_match_alone_and_reference():
    # uneven sizes, seeds, bath rates and adaptation strengths, two golden cases
    cfgs = [CASES["small_1x1"](), small(3, 2, ms=300, seed=11, nu_ext_hz=4.0, alpha_c=0.5),
            CASES["small_2x2"](), small(1, 2, ms=300, seed=5, nu_ext_hz=2.0, alpha_c=1.8)]
    together, ev_together = rasters_stepped_together(cfgs, 300)
    for c, (ids, ts), ev in zip(cfgs, together, ev_together):
        alone, ev_alone = rasters_stepped_together([c], 300)
        np.testing.assert_array_equal(ids, alone[0][0])
        np.testing.assert_array_equal(ts, alone[0][1])
        assert ev == ev_alone[0]
    for k, name in ((0, "small_1x1"), (2, "small_2x2")):
        gi, gt = gio.raster(name)
        np.testing.assert_array_equal(together[k][0], gi)
        np.testing.assert_array_equal(together[k][1], gt)


def test_graph_runs_match_plain_steps():
    """The batched graph (dpsnn_graph_create/run, 80 steps of every network
    per run) gives each network the raster and event count of dpsnn_step,
    with the launch shapes the autotuner may choose, and refuses a run at a
    step other than the one it was recorded at."""
    import importlib
    B = importlib.import_module(E.__name__.rsplit(".", 1)[0] + ".batch")
    cfgs = [CASES["small_1x1"](), CASES["small_2x2"](), small(3, 2, ms=300, seed=11, nu_ext_hz=4.0, alpha_c=0.5,
                                                              glob_h=6)]
    plain, ev_plain = rasters_stepped_together(cfgs, 241)
    engines = [E.Engine(c) for c in cfgs]
    for e, c, bpm in zip(engines, cfgs, (4, 16, 0)):   # uneven grids, defaults on the last
        e.set_launch_shape(*B.shape_rule(bpm)(e, c))
        e.step(1)
    out = [([], []) for _ in cfgs]
    for e, (ids, ts) in zip(engines, out):
        i, t = e.spikes(0)
        ids.append(i)
        ts.append(t)
    g = E.Graph(engines, 80)
    for run in range(3):
        g.run()
        for e, (ids, ts) in zip(engines, out):
            for t in range(1 + 80 * run, 81 + 80 * run):
                i, tt = e.spikes(t)
                ids.append(i)
                ts.append(tt)
    for (ids, ts), (pi, pt), e, ev in zip(out, plain, engines, ev_plain):
        np.testing.assert_array_equal(np.concatenate(ids), pi)
        np.testing.assert_array_equal(np.concatenate(ts), pt)
        assert e.events_delivered() == ev and e.time_ms == 241
    engines[0].step(1)   # now at step 242: not the recorded step modulo 80
    with pytest.raises(E.EngineError, match="recorded at"):
        g.run()
    g.close()
    for e in engines:
        e.close()
