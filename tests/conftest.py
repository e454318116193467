import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(ROOT, "tests", "golden", "reference_golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import cfdrs_b200._lib as L
    L.load()
    return torch


# Under `pytest -x` the first failure ends the run, so the suites of the solve
# path itself (parity, GMRES, batch, adjoint, recompute) run before the
# components added on top of them (device network assembly, the saddle-point
# tiers, the pressure dispatch), then the wait-timeout check, and the no-alloc
# entry point's test runs last of all.
_FILE_ORDER = ["test_gpu_parity", "test_gpu_configs", "test_gpu_gmres", "test_gpu_batch", "test_gpu_network_cascade", "test_gpu_adjoint", "test_gpu_recompute",
               "test_gpu_network_assembly", "test_gpu_simple", "test_gpu_component", "test_gpu_pressure",
               "test_zy_wait_timeout", "test_zz_no_alloc"]


def pytest_collection_modifyitems(session, config, items):
    def rank(item):
        stem = os.path.splitext(os.path.basename(str(item.fspath)))[0]
        return _FILE_ORDER.index(stem) if stem in _FILE_ORDER else -1
    items.sort(key=rank)  # stable: CPU suites (rank -1) first, in their collected order
