"""Host side of the engine: C ABI exports and the env/ini parser (no GPU)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from tests.conftest import ROOT, engine_module
from tests.golden.cases import CASES

E = engine_module()
HEADER = os.path.join(ROOT, "include", "dpsnn_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(dpsnn_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = E.load_library()
    missing = [f for f in declared_functions() if not hasattr(lib, f)]
    assert not missing, missing


def test_localnet_exports_the_dal_trio_with_cxx_linkage():
    """libdpsnn_localnet.so defines the three symbols the reference's MPI
    main leaves undefined (C++ names of localNetProcess.h:72-74)."""
    lib = C.CDLL(os.path.join(ROOT, "201812realtimecortsim_b200", "libdpsnn_localnet.so"))
    for sym in ("_Z20localNetProcess_initP8_process", "_Z20localNetProcess_fireP8_process",
                "_Z22localNetProcess_finishP8_process", "_Z13getParametersj"):
        assert hasattr(lib, sym), sym


def test_localnet_getparameters_reads_the_run_inputs(tmp_path, monkeypatch):
    """getParameters(loc_h) (C++ name of DPSNN_getParameters.h:7) parses the
    env_* variables and the input files of the current directory."""
    cfg = CASES["small_2x2"]()
    _env_for(cfg, tmp_path, monkeypatch)
    monkeypatch.chdir(tmp_path)
    lib = C.CDLL(os.path.join(ROOT, "201812realtimecortsim_b200", "libdpsnn_localnet.so"))
    f = lib._Z13getParametersj
    f.restype = E.Params
    f.argtypes = [C.c_uint32]
    got = f(0)
    want = E.params_from_env(str(tmp_path)).p
    for field in ("cfx", "cfy", "glob_h", "D", "nsub", "global_seed", "stencil_dim"):
        assert getattr(got, field) == getattr(want, field), field
    assert list(got.count) == list(want.count)


def test_binding_covers_the_header():
    assert set(declared_functions()) <= set(E.EXPORTS)


def _env_for(cfg, workdir, monkeypatch):
    env = cfg.write(str(workdir))
    for k, v in env.items():
        monkeypatch.setenv(k, v)


def _delay_range_grid():
    from tests.conftest import netconfig
    return netconfig().cortical_grid(6, 6, total_ms=100, glob_h=12, delay_range_subpop=True)


@pytest.mark.parametrize("name", ["small_2x2", "small_2x2_stdp", "c1_2x2", "delay_range_6x6"])
def test_parser_reads_what_netconfig_writes(name, tmp_path, monkeypatch):
    # delay_range_6x6: a fourth, empty sub-population widening the delay range
    cfg = _delay_range_grid() if name == "delay_range_6x6" else CASES[name]()
    _env_for(cfg, tmp_path, monkeypatch)
    got = E.params_from_env(str(tmp_path))
    want = E.params_from_netconfig(cfg)
    for field, _ in E.Params._fields_:
        if field in ("spec", "bath"):
            continue
        a, b = getattr(got.p, field), getattr(want.p, field)
        if hasattr(a, "__len__"):
            assert list(a) == list(b), field
        elif field not in ("moduloSec", "ratesSampling", "startStatFiles_s", "stopStatFiles_s",
                           "startRatesPerPop_s", "stopRatesPerPop_s", "howManyOutputFiles",
                           "spikes_writeDisable", "statRatesPerPop_writeDisable"):
            assert a == b, field
    np.testing.assert_array_equal(got.spec, want.spec.reshape(-1))
    np.testing.assert_array_equal(got.bath, want.bath.reshape(-1))


def test_parser_reports_missing_variable(tmp_path, monkeypatch):
    cfg = CASES["small_1x1"]()
    _env_for(cfg, tmp_path, monkeypatch)
    monkeypatch.delenv("env_D")
    with pytest.raises(E.EngineError, match="env_D"):
        E.params_from_env(str(tmp_path))


def test_parser_reports_missing_file(tmp_path, monkeypatch):
    cfg = CASES["small_1x1"]()
    _env_for(cfg, tmp_path, monkeypatch)
    os.remove(tmp_path / "connectivity.txt")
    with pytest.raises(E.EngineError, match="connectivity.txt"):
        E.params_from_env(str(tmp_path))


def test_parser_applies_reference_build_limits(tmp_path, monkeypatch):
    cfg = CASES["c1_2x2"]()
    _env_for(cfg, tmp_path, monkeypatch)
    monkeypatch.setenv("env_CFX", "24")
    monkeypatch.setenv("env_CFY", "24")
    with pytest.raises(E.EngineError, match="too many neurons"):
        E.params_from_env(str(tmp_path))      # 720000 neurons on one rank > miniLocN
    monkeypatch.setenv("DPSNN_MAX_LOC_N", "1000000")
    E.params_from_env(str(tmp_path))


def _has_gpu():
    try:
        cudart = C.CDLL("libcudart.so")
    except OSError:
        return False
    n = C.c_int(0)
    return cudart.cudaGetDeviceCount(C.byref(n)) == 0 and n.value > 0


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU failure path")
def test_create_fails_loudly_without_gpu():
    with pytest.raises(E.EngineError, match="CUDA"):
        E.Engine(CASES["small_1x1"]())
