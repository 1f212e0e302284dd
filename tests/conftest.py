import importlib
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def package():
    return importlib.import_module("201812realtimecortsim_b200")


def netconfig():
    return importlib.import_module("201812realtimecortsim_b200.netconfig")


def engine_module():
    return importlib.import_module("201812realtimecortsim_b200.engine")
