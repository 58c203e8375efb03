"""Shared test set-up: import paths, the ``gpu`` marker, small graph helpers."""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "cbm-gpu_b200")
for p in (PKG, REPO):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def pytest_collection_modifyitems(config, items):
    # a GPU test on a machine without a GPU fails loudly instead of skipping
    pass


def random_graph(n, avg_deg, seed, symmetric=True, self_loops=False, isolated=0):
    """Random binary graph as coalesced int32 edge_index."""
    from cbm.synthetic import coalesce_symmetric

    rng = np.random.Generator(np.random.PCG64(seed))
    m = int(n * avg_deg / (2 if symmetric else 1))
    # isolated nodes are ids [n//4, n//4 + isolated): inside the index range
    active_ids = np.setdiff1d(np.arange(n), np.arange(n // 4, n // 4 + isolated))
    active = active_ids.size
    r = active_ids[rng.integers(0, active, m)]
    c = active_ids[rng.integers(0, active, m)]
    r[0], c[0] = 0, n - 1  # both ends present, so that max(index) + 1 == n
    if symmetric:
        ei = coalesce_symmetric(r, c, n)
    else:
        keep = self_loops | (r != c)
        key = np.unique(r[keep].astype(np.int64) * n + c[keep])
        ei = np.stack([key // n, key % n]).astype(np.int32)
    if self_loops and symmetric:
        extra = active_ids[::3]
        key = np.unique(np.concatenate([ei[0].astype(np.int64) * n + ei[1], extra * n + extra]))
        ei = np.stack([key // n, key % n]).astype(np.int32)
    return ei


def near_dup_graph(n, seed, frac=0.4, flip=0.1, deg=10):
    """Rows that are flipped copies of other rows: deep-ish CBM trees."""
    from cbm.synthetic import community_graph, near_duplicates

    rng = np.random.Generator(np.random.PCG64(seed))
    ei = community_graph(n, 32, deg, 2, rng=rng)
    return near_duplicates(ei, n, frac, flip, rng=rng)


def chain_graph(n):
    """Rows 0..n-1 where row i = {0..i}: every row is its predecessor plus one
    column, so the CBM tree is one long chain."""
    rows, cols = [], []
    for i in range(n):
        for j in range(i + 1):
            rows.append(i)
            cols.append(j + n)  # columns n..2n-1 so that there are no self loops
    # square matrix of size 2n: the last n rows are empty
    return np.array([rows, cols], dtype=np.int32), 2 * n


@pytest.fixture(scope="session")
def lib():
    from cbm import _lib

    return _lib.load()


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle

    oracle.lib()
    return oracle
