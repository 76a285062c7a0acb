"""Shared fixtures: the `gpu` marker, the package loader and the oracle loader.

`-m "not gpu"` tests need no GPU: they cover the oracle against the golden vectors, the host-side
policy and validation logic, the multi-rank sharding on gloo, and that the C-ABI library loads and
exports every declared symbol.  `-m gpu` tests call the CUDA path through the C ABI and compare it
with the oracle.
"""
from __future__ import annotations

import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# The mixed-degree tuner's file stays out of the test session: tests tune on a few instances,
# choices a later batch of hundreds should not inherit.  (The test of the file itself sets its own.)
os.environ.setdefault("EGG_TUNE_CACHE", "")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libeggman_b200.so")


def load_package():
    """Import theeggman.jl_b200/ under the module name `theeggman_b200`."""
    if "theeggman_b200" in sys.modules:
        return sys.modules["theeggman_b200"]
    d = os.path.join(ROOT, "theeggman.jl_b200")
    spec = importlib.util.spec_from_file_location("theeggman_b200", os.path.join(d, "__init__.py"),
                                                  submodule_search_locations=[d])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["theeggman_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def egg():
    return load_package()


@pytest.fixture(scope="session")
def W(egg):
    """Seeded workload generators (theeggman.jl_b200/workloads.py)."""
    from theeggman_b200 import workloads

    return workloads


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle as O

    O.build()
    return O


@pytest.fixture(scope="session")
def golden():
    import json

    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        return json.load(f)


def dec(x):
    """Decode a fixture number: a hex float string, or [re, im] hex pair."""
    if isinstance(x, list):
        return complex(float.fromhex(x[0]), float.fromhex(x[1]))
    return float.fromhex(x)


def dec_matrix(rows):
    import numpy as np

    vals = [[dec(v) for v in r] for r in rows]
    cplx = any(isinstance(v, complex) for r in vals for v in r)
    return np.array(vals, dtype=np.complex128 if cplx else np.float64)
