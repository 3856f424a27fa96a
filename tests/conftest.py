"""Shared fixtures. GPU tests are marked `gpu`; everything else runs on the CPU."""
import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def mp():
    """The product package (imports libmp.so; fails loudly if it is missing)."""
    return importlib.import_module("2017multiphase_b200")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.build()
    return oracle


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def refhost():
    """The reference's own kernels compiled for the host (oracle/make_refhost.py),
    built once per session from the reference tree; tests that use it skip
    themselves when the tree is absent."""
    from oracle import make_refhost
    make_refhost.build(make_refhost.DEFAULT_SRC, quiet=True)
    from oracle import refhost as rh
    return rh
