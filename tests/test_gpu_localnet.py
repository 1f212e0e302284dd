"""The DAL process trio (libdpsnn_localnet.so) as a drop-in: run through a
single-process main, its output files are byte-identical to the reference's
(spikes, ratesPerPop and FiringsInChronoWindow files of the golden runs)."""
import hashlib
import os
import subprocess

import pytest

from tests.golden import io as gio
from tests.golden.cases import CASES

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUNNER = os.path.join(ROOT, "201812realtimecortsim_b200", "dpsnn_localnet_run")
# the reference's own MPI main (DPSNN_mainUnderMPI.c) linked against the
# trio, built by `make -C oracle dropin` where the reference sources exist
REF_MAIN = os.path.join(ROOT, "oracle", "_ref", "dpsnn_ref_main_dropin")


def sha256(path):
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def run_in(binary, cfg, workdir):
    env = dict(os.environ)
    env.update(cfg.write(workdir))
    r = subprocess.run([binary], cwd=workdir, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "ERROR" not in r.stdout, r.stdout[-2000:]
    return r.stdout


@pytest.mark.parametrize("name", sorted(CASES))
def test_trio_output_files_identical_to_reference(name, tmp_path):
    cfg = CASES[name]()
    out = run_in(RUNNER, cfg, str(tmp_path))
    assert "total fire time" in out
    want = gio.manifest()[name]["outputs_sha256"]
    got = {fn: sha256(os.path.join(tmp_path, fn)) for fn in want if os.path.exists(os.path.join(tmp_path, fn))}
    assert got == want


@pytest.mark.skipif(not os.path.exists(REF_MAIN), reason="reference main not linked here")
def test_reference_main_over_trio(tmp_path):
    cfg = CASES["small_2x2"]()
    out = run_in(REF_MAIN, cfg, str(tmp_path))
    assert "total fire time" in out
    want = gio.manifest()["small_2x2"]["outputs_sha256"]
    for fn, h in want.items():
        assert sha256(os.path.join(tmp_path, fn)) == h, fn


def test_trio_writes_every_emulated_rank(tmp_path):
    """With env_globH=4 the trio writes the four ranks' spike files: each
    holds only its rank's neurons, and together they are the raster of the
    restatement run with the same four ranks."""
    import dpsnn_oracle as O
    cfg = CASES["small_2x2"]()
    cfg.glob_h = 4
    cfg.total_ms = 200
    run_in(RUNNER, cfg, str(tmp_path))
    got = []
    for h in range(4):
        with open(os.path.join(tmp_path, f"spikes-sec0-C4-H4-h{h:03d}.dat")) as f:
            rows = [line.split() for line in f]
        assert all(h * 100 <= int(a) < (h + 1) * 100 for a, _ in rows)
        got += [(int(a), b) for a, b in rows]
    orc = O.OracleNet(cfg, 1)
    want = []
    for _ in range(cfg.total_ms):
        ids, ts = orc.step()
        want += [(int(i), "%.7g" % t) for i, t in zip(ids, ts)]
    assert len(want) > 0
    assert sorted(got) == sorted(want)


@pytest.mark.parametrize("name", [n for n, e in sorted(gio.manifest().items()) if "probe_sha256" in e])
def test_trio_plasticity_side_files_identical_to_reference(name, tmp_path):
    """With the synapse probe and STDP event switches on, the trio writes rank
    0's synPeriodicProbe_A/B files (synapses before and after each x999 ms
    plasticity update) and its STDPevent files (every causal and anti-causal
    contribution between rank-0 neurons, in the reference's order), byte for
    byte as the reference does; the other output files stay identical too."""
    cfg = CASES[name]()
    cfg.extra_env.update({"env_statSynPeriodicProbe_writeDisable": "0",
                          "env_startSynPeriodicProbe_s": "0",
                          "env_stopSynPeriodicProbe_s": "100000",
                          "env_statSTDPevent_writeDisable": "0",
                          "env_startSTDPevent_s": "0",
                          "env_stopSTDPevent_s": "100000"})
    run_in(RUNNER, cfg, str(tmp_path))
    entry = gio.manifest()[name]
    want = dict(entry["probe_sha256"], **entry["stdp_event_sha256"], **entry["outputs_sha256"])
    side = sorted(fn for fn in os.listdir(tmp_path) if fn.startswith(("synPeriodicProbe_", "STDPevent-")))
    assert side == sorted(list(entry["probe_sha256"]) + list(entry["stdp_event_sha256"]))
    got = {fn: sha256(os.path.join(tmp_path, fn)) for fn in want if os.path.exists(os.path.join(tmp_path, fn))}
    assert got == want
