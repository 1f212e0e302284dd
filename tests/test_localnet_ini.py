"""The Perseo .ini description the trio writes at init (DPSNN_WRITE_INI_FILES=1)
is byte-identical to the reference's writeIniFiles output.  The files are
written before the engine is built, so this runs on a machine without a GPU
too (there, init then stops with the reference's ERROR exit)."""
import hashlib
import os
import subprocess

import pytest

from tests.golden import io as gio
from tests.golden.cases import CASES

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUNNER = os.path.join(ROOT, "201812realtimecortsim_b200", "dpsnn_localnet_run")


@pytest.mark.parametrize("name", [n for n, e in sorted(gio.manifest().items()) if "ini_sha256" in e])
def test_ini_files_identical_to_reference(name, tmp_path):
    cfg = CASES[name]()
    cfg.total_ms = 10
    env = dict(os.environ)
    env.update(cfg.write(str(tmp_path)))
    env["DPSNN_WRITE_INI_FILES"] = "1"
    subprocess.run([RUNNER], cwd=tmp_path, env=env, capture_output=True, text=True, timeout=600)
    want = gio.manifest()[name]["ini_sha256"]
    assert want
    for fn, h in want.items():
        with open(os.path.join(tmp_path, fn), "rb") as f:
            assert hashlib.sha256(f.read()).hexdigest() == h, fn
