import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def song():
    """The product package (its directory name starts with a digit)."""
    return importlib.import_module("2020_song_ex_b200")


@pytest.fixture(scope="session")
def ds():
    return importlib.import_module("2020_song_ex_b200.datasets")


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    return o


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a -m gpu test ran without a CUDA device")
    return torch


def knn_graph(data: np.ndarray, block_size: int, degree: int, seed: int = 0,
              drop: float = 0.1) -> np.ndarray:
    """A small test graph: each node's `degree` nearest neighbours, with some
    slots emptied (-1) and the rest shuffled, so rows hold holes anywhere."""
    rng = np.random.default_rng(seed)
    x = data.astype(np.float64)
    sq = (x * x).sum(1)
    d = sq[:, None] - 2.0 * x @ x.T + sq[None, :]
    np.fill_diagonal(d, np.inf)
    nn = np.argsort(d, axis=1, kind="stable")[:, :degree].astype(np.int32)
    adj = np.full((data.shape[0], block_size), -1, np.int32)
    adj[:, :degree] = nn
    mask = rng.random(adj.shape) < drop
    adj[mask] = -1
    for r in adj:
        rng.shuffle(r)
    return adj
