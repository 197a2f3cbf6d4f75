"""Shared test setup: import paths, the `gpu` marker, seeded matrices."""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(REPO, "matrix-reorder_b200"), os.path.join(REPO, "oracle"), REPO):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def M():
    import mrb200
    mrb200.lib()
    mrb200.gen()
    return mrb200


@pytest.fixture(scope="session")
def O():
    import pyoracle
    pyoracle.orc()
    return pyoracle


def csr_from_dense_pattern(rows):
    """CSR from a list of column lists (values deterministic)."""
    rp = np.zeros(len(rows) + 1, np.int32)
    for i, r in enumerate(rows):
        rp[i + 1] = rp[i] + len(r)
    ci = np.array([c for r in rows for c in r], np.int32)
    v = ((np.arange(ci.size) % 13) - 6).astype(np.float32) / 4.0
    return rp, ci, v


def csr_random(n, nnz_per_row_max, seed, ncols=None, empty_frac=0.0):
    """Random CSR with sorted unique columns per row."""
    rng = np.random.default_rng(seed)
    ncols = n if ncols is None else ncols
    rows = []
    for _ in range(n):
        k = 0 if rng.random() < empty_frac else int(rng.integers(0, nnz_per_row_max + 1))
        k = min(k, ncols)
        rows.append(sorted(rng.choice(ncols, size=k, replace=False).tolist()))
    rp, ci, _ = csr_from_dense_pattern(rows)
    v = rng.uniform(-1, 1, ci.size).astype(np.float32)
    return rp, ci, v
