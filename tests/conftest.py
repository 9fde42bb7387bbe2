"""Shared fixtures.  Tests marked `gpu` need a B200 and the built library;
everything else runs on CPU (oracle, golden fixtures, host logic, ABI)."""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libpiro_b200.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def golden_grids():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        man = json.load(f)
    out = []
    for g in man["grids"]:
        out.append((tuple(g["n"]), dict(np.load(os.path.join(GOLDEN, g["file"])))))
    return out


@pytest.fixture(scope="session")
def golden_hashes():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)["hashes"]


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("GPU test run without a CUDA device")
    from piro_b200 import _lib
    _lib.lib()
    return torch


def f32_bits_equal(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))
