"""Test configuration: the `gpu` marker, golden-fixture loading and oracle access.

`-m "not gpu"` runs on any machine (oracle vs golden fixtures, host logic, the C ABI
symbol table); `-m gpu` runs the CUDA parity tests against the oracle and the fixtures.
"""

import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")
    config.addinivalue_line("markers", "slow: long-running case")


def pytest_collection_modifyitems(config, items):
    try:
        import torch

        has_cuda = torch.cuda.is_available()
    except Exception:  # pragma: no cover
        has_cuda = False
    if has_cuda:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def golden(name: str):
    path = os.path.join(GOLDEN, f"{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"golden fixture {name}.npz not generated")
    return np.load(path)


def cases(g):
    """Iterate the c{k}_ prefixed cases of a golden archive as dicts."""
    out = []
    for k in range(int(g["count"])):
        p = f"c{k}_"
        out.append({key[len(p):]: g[key] for key in g.files if key.startswith(p)})
    return out


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.build()
    return O
