"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on CPU."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def golden_state(g):
    from activechi4_b200.init import State
    return State(float(g["L"]), g["x"].copy(), g["xu"].copy(), g["p"].copy(), g["type"].copy(),
                 g["act_tag"].copy(), g["k"].copy())


@pytest.fixture(scope="session")
def g1000():
    return load_golden("ka_n1000.npz")


@pytest.fixture(scope="session")
def g4000():
    return load_golden("ka_n4000.npz")


@pytest.fixture(scope="session")
def g500():
    return load_golden("ka_n500.npz")


@pytest.fixture(scope="session")
def sched():
    return load_golden("schedule.npz")


@pytest.fixture(scope="session")
def cuda_lib():
    """The in-tree CUDA library, (re)built if its sources are newer."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from activechi4_b200 import build
    build.build()
    from activechi4_b200 import _abi
    return _abi.lib()


def force_err(F, Fref):
    """max_i |F_i - Fref_i| / rms |Fref|"""
    rms = np.sqrt((Fref ** 2).sum(axis=1).mean())
    return np.abs(F - Fref).max() / rms


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)
