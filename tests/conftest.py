"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on a CPU-only machine.

The oracle (oracle/) is the checker: tests import it to build reference models and
expected results.  The product path under test is h2_b200 (libh2g.so, sm_100a).
"""
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than ~20 s on 8 CPU cores")


def golden(name):
    with open(os.path.join(GOLDEN, name)) as fh:
        return json.load(fh)


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


_MODELS = {}


def mode3_model(O, NX, NY=None, NZ=30, **kw):
    """Oracle-built Mode-3 model (cached per session); returns a fresh copy of the arrays."""
    import copy
    NY = NX if NY is None else NY
    key = (NX, NY, NZ, tuple(sorted(kw.items())))
    if key not in _MODELS:
        _MODELS[key] = O.build_mode3(NX, NY, NZ, threads=os.cpu_count(), **kw)
    return copy.deepcopy(_MODELS[key])


@pytest.fixture(scope="session")
def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
