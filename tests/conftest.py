import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (runs the CUDA library)")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def golden_vecs():
    return dict(np.load(os.path.join(GOLDEN, "golden_vectors.npz")))


def terms_from_golden(m):
    return [(complex(c[0], c[1]), [(op, s) for op, s in f]) for c, f in m["terms"]]


def dense_from_coo(rows, cols, vals, dim):
    """Sum duplicate entries in the reference's order (its SpMV row sum)."""
    H = np.zeros((dim, dim), dtype=np.complex128)
    for r, c, v in zip(rows, cols, vals):
        H[r, c] += v
    return H
