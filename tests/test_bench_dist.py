"""bench.py's multi-process harness on CPU: two ranks launched by
torch.distributed.run with the gloo backend run the reference arm; rank 0
alone measures and prints one JSON line, the other rank exits cleanly.  The
network is a 2x2 grid run by the reference as 2 MPI processes (the arm's
path for the 24x24 benchmark with 192, on a size that runs in seconds)."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "dpsnn_ref_mp")),
                    reason="reference binary not built")
def test_reference_arm_two_ranks_gloo():
    env = dict(os.environ)
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "4", "--warmup", "20",
           "--grid", "2x2", "--ranks", "2"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    out = lines[0]
    assert out["impl"] == "reference" and out["n_gpus"] == 2
    assert out["value"] > 0 and out["e2e"]["value"] == out["value"]
    assert out["cpu_baseline"]["kind"] == "reference"
    assert out["config"]["timed_steps"] == [20, 23] and out["config"]["events_per_step"] > 0
