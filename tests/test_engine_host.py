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


def test_entry_points_reject_null_arguments():
    """Every entry point that takes an engine, a graph or an output pointer
    checks it before it touches the device: DPSNN_E_PARAM (-1) with a message,
    0 from the accessors, nothing from the destructors."""
    lib = E.load_library()
    E_PARAM = -1
    u32 = C.c_uint32(0)
    P = C.c_void_p
    calls = {
        "dpsnn_create": lambda: lib.dpsnn_create(None, None, None),
        "dpsnn_step": lambda: lib.dpsnn_step(None, 1),
        "dpsnn_sync": lambda: lib.dpsnn_sync(None),
        "dpsnn_step_many": lambda: lib.dpsnn_step_many(None, 2, 1),
        "dpsnn_spikes": lambda: lib.dpsnn_spikes(None, 0, None, None, 0, C.byref(u32)),
        "dpsnn_spikes_range": lambda: lib.dpsnn_spikes_range(None, 0, 1, None, None, 0, None),
        "dpsnn_rank_spikes_noalloc": lambda: lib.dpsnn_rank_spikes_noalloc(None, 0, 0, None, None, 0, C.byref(u32)),
        "dpsnn_state": lambda: lib.dpsnn_state(None, None, None, None, None, None),
        "dpsnn_bath_params": lambda: lib.dpsnn_bath_params(None, None, None),
        "dpsnn_backward_synapses": lambda: lib.dpsnn_backward_synapses(None, 0, None, None, None, None, None, None),
        "dpsnn_enable_ltp_probe": lambda: lib.dpsnn_enable_ltp_probe(None),
        "dpsnn_ltp_probe": lambda: lib.dpsnn_ltp_probe(None, 0, None, None, None, None, None),
        "dpsnn_enable_stdp_events": lambda: lib.dpsnn_enable_stdp_events(None),
        "dpsnn_stdp_events": lambda: lib.dpsnn_stdp_events(None, None, None, None, None, 0, C.byref(u32)),
        "dpsnn_set_timing": lambda: lib.dpsnn_set_timing(None, 1),
        "dpsnn_kernel_times": lambda: lib.dpsnn_kernel_times(None, None, None),
        "dpsnn_graph_run": lambda: lib.dpsnn_graph_run(None),
        "dpsnn_set_launch_shape": lambda: lib.dpsnn_set_launch_shape(None, 0, 0, 0),
    }
    for name, call in calls.items():
        assert call() == E_PARAM, name
        assert lib.dpsnn_last_error(), name
    for name in ("dpsnn_glob_n", "dpsnn_time_ms", "dpsnn_synapse_count", "dpsnn_events_delivered",
                 "dpsnn_device_bytes", "dpsnn_kernel_launches"):
        assert getattr(lib, name)(None) == 0, name
    assert lib.dpsnn_rank_synapse_count(None, 0) == 0
    assert lib.dpsnn_cuda_stream(None) is None
    lib.dpsnn_destroy(None)
    lib.dpsnn_graph_destroy(None)
    # a graph holds a positive multiple of the 80 ring slots of at least one
    # engine; these are refused before any engine is read
    g = P()
    assert lib.dpsnn_graph_create(None, 0, 80, C.byref(g)) == E_PARAM and not g.value
    eng = (P * 1)(None)
    assert lib.dpsnn_graph_create(eng, 1, 40, C.byref(g)) == E_PARAM and not g.value
    assert b"multiple of 80" in lib.dpsnn_last_error()
    assert lib.dpsnn_graph_create(eng, 1, 80, C.byref(g)) == E_PARAM
    assert b"null engine 0" in lib.dpsnn_last_error()
    assert lib.dpsnn_step_many(eng, 1, 1) == E_PARAM
    assert b"null engine 0" in lib.dpsnn_last_error()
