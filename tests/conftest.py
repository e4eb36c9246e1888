"""Shared pytest configuration: the `gpu` marker and data builders."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (B200) device")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def load_golden(name):
    with np.load(os.path.join(GOLDEN, name)) as f:
        return {k: f[k] for k in f.files}


def make_set(nm, ma, rep, n_species, seed, n_min=1, species=None):
    """Random-normal descriptors with ragged atom counts (the style of the
    reference's unit tests)."""
    rng = np.random.default_rng(seed)
    sp = np.asarray(species if species is not None else np.arange(1, n_species + 1), np.int32)
    X = rng.standard_normal((nm, ma, rep))
    N = rng.integers(n_min, ma + 1, size=nm).astype(np.int32)
    Q = np.zeros((nm, ma), np.int32)
    for a in range(nm):
        Q[a, :N[a]] = rng.choice(sp, size=N[a])
    dX = rng.standard_normal((nm, ma, rep, 3 * ma))
    return X, dX, Q, N
