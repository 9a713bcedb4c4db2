import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long CPU test")


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle
    oracle.lib()
    return oracle


def _load_product():
    import importlib.util
    path = os.path.join(ROOT, "fluid-simulation-app_b200", "fluidcu.py")
    spec = importlib.util.spec_from_file_location("fluidcu", path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules["fluidcu"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def fcu():
    mod = _load_product()
    mod.lib()
    return mod


@pytest.fixture(scope="session")
def wl():
    import importlib.util
    path = os.path.join(ROOT, "fluid-simulation-app_b200", "workloads.py")
    spec = importlib.util.spec_from_file_location("workloads", path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules["workloads"] = mod
    spec.loader.exec_module(mod)
    return mod
