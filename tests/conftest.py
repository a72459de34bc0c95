import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "parareal-cc-cfv-split-gpu_b200"
for p in (ROOT / "oracle", PKG, ROOT / "tests" / "golden"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libccfv.so")
    config.addinivalue_line("markers", "slow: long-running")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def ccfv():
    import ccfv as M
    M.lib()
    return M


def seeded_field(N, seed, ny=None, domain=(-1.0, 1.0, -1.0, 1.0)):
    """Smooth random field, non-zero on the boundary, plus noise."""
    ny = N if ny is None else ny
    rng = np.random.default_rng(seed)
    x = domain[0] + (np.arange(N) + 0.5) * ((domain[1] - domain[0]) / N)
    y = domain[2] + (np.arange(ny) + 0.5) * ((domain[3] - domain[2]) / ny)
    X, Y = np.meshgrid(x, y, indexing="ij")
    f = 0.2 + 0.1 * X - 0.05 * Y
    sx, sy = domain[1] - domain[0], domain[3] - domain[2]
    for _ in range(4):
        cx = rng.uniform(domain[0] + 0.1 * sx, domain[1] - 0.1 * sx)
        cy = rng.uniform(domain[2] + 0.1 * sy, domain[3] - 0.1 * sy)
        w = rng.uniform(0.05, 0.3) * sx * sy / 4
        a = rng.uniform(0.3, 1.0)
        f = f + a * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / w)
    f = f + 1e-3 * rng.standard_normal((N, ny))
    return np.ascontiguousarray(f)


def periodic_field(N, seed, ny=None):
    """Smooth periodic field on [0,1]^2 (Fourier modes) plus a Gaussian bump."""
    ny = N if ny is None else ny
    rng = np.random.default_rng(seed)
    x = (np.arange(N) + 0.5) / N
    y = (np.arange(ny) + 0.5) / ny
    X, Y = np.meshgrid(x, y, indexing="ij")
    f = 1.0 + 0.0 * X
    for kx in range(0, 3):
        for ky in range(-2, 3):
            a, b = rng.normal(0, 0.2, 2)
            f = f + a * np.cos(2 * np.pi * (kx * X + ky * Y)) + b * np.sin(2 * np.pi * (kx * X + ky * Y))
    return np.ascontiguousarray(f)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))
