"""Shared test setup: the `gpu` marker, the package and the CPU oracle.

Tests marked `gpu` need a CUDA device and the built libkrv_gpu.so; the rest
run on the CPU (oracle against golden vectors, host logic, library exports).
"""
import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
ORACLE_DIR = os.path.join(ROOT, "oracle")
if ORACLE_DIR not in sys.path:
    sys.path.insert(0, ORACLE_DIR)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libkrv_gpu.so")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O  # noqa: E402  (oracle/oracle.py, test infrastructure)
    O.lib()
    return O


@pytest.fixture(scope="session")
def kb():
    return importlib.import_module("krishiv-engine_b200")


@pytest.fixture(scope="session")
def rt(kb):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    r = kb.Runtime.on_torch_stream(0)
    yield r
    r.synchronize()
