import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA path through the C ABI")
    config.addinivalue_line("markers", "slow: long-running case")


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def uniform_system(n, seed, cell=None, charges="pm1"):
    """Seeded synthetic system: fractional-uniform positions, neutral charges."""
    rng = np.random.default_rng(seed)
    cell = np.eye(3) if cell is None else np.asarray(cell, dtype=np.float64)
    frac = rng.uniform(0.0, 1.0, (n, 3))
    pos = frac @ cell.T
    if charges == "pm1":
        q = np.ones(n)
        q[: n // 2] = -1.0
        rng.shuffle(q)
        q -= q.mean()
    else:
        q = rng.uniform(-1.0, 1.0, n)
        q -= q.mean()
    return cell, pos, q


def clustered_system(n, seed, cell, n_clusters=8, sigma=0.01):
    """Half fractional-uniform, half Gaussian clusters (Cartesian sigma), wrapped into the cell."""
    rng = np.random.default_rng(seed)
    cell = np.asarray(cell, dtype=np.float64)
    inv = np.linalg.inv(cell)
    nu = n // 2
    frac_u = rng.uniform(0, 1, (nu, 3))
    centers = rng.uniform(0, 1, (n_clusters, 3)) @ cell.T
    which = rng.integers(0, n_clusters, n - nu)
    pts = centers[which] + rng.normal(0, sigma, (n - nu, 3))
    frac_c = (pts @ inv.T) % 1.0
    frac = np.vstack([frac_u, frac_c])
    pos = frac @ cell.T
    q = np.ones(n)
    q[: n // 2] = -1.0
    rng.shuffle(q)
    q -= q.mean()
    return cell, pos, q


TRICLINIC = np.array([[1.0, 0.3, 0.2], [0.0, 0.9, 0.25], [0.0, 0.0, 0.85]])  # columns a1, a2, a3
