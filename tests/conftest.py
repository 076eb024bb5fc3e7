"""Shared fixtures.  Tests marked `gpu` need a CUDA device and the in-tree
libsph_b200.so; everything else runs on the CPU (the oracle, the golden
fixtures, the host-side logic and the library's symbol table)."""
from __future__ import annotations

import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")


@pytest.fixture(scope="session")
def pkg():
    return importlib.import_module("real-time-planetary-impacts-mps_b200")


@pytest.fixture(scope="session")
def O():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def eos_paths(pkg):
    return pkg.eos_tables.ensure_tables()


@pytest.fixture(scope="session")
def eos_grids(O, eos_paths):
    return (O.aneos_load(eos_paths["forsterite"], 2048), O.aneos_load(eos_paths["Fe85Si15"], 2048))


def golden(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, name)) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def cuda(pkg):
    """Skip when no CUDA device is visible; fail when the library is missing."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    pkg.build()
    return pkg._lib.load()
