import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the product kernels")


def reference_root():
    """Where the reference source tree lies: $REF, else the default of oracle/Makefile's REF."""
    if os.environ.get("REF"):
        return os.environ["REF"]
    for line in open(os.path.join(ROOT, "oracle", "Makefile")):
        if line.startswith("REF ?="):
            return line.split("?=", 1)[1].strip()
    return ""


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def port_oracle():
    from oracle.oracle import Oracle
    return Oracle("port")
