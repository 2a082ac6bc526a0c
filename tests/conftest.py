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


def batch_cell(rng):
    """Triclinic cell of the many-systems workload: lengths U[0.8, 1.2], angles
    U[75, 105] degrees, a1 along x, a2 in the xy plane (columns = vectors)."""
    L = rng.uniform(0.8, 1.2, 3)
    al, be, ga = np.radians(rng.uniform(75.0, 105.0, 3))
    a1 = np.array([L[0], 0.0, 0.0])
    a2 = L[1] * np.array([np.cos(ga), np.sin(ga), 0.0])
    cx = np.cos(be)
    cy = (np.cos(al) - np.cos(be) * np.cos(ga)) / np.sin(ga)
    a3 = L[2] * np.array([cx, cy, np.sqrt(max(1.0 - cx * cx - cy * cy, 1e-12))])
    return np.column_stack([a1, a2, a3])


def batch_systems(nsys, seed, n_min=1000, n_max=100000):
    """nsys systems: N log-uniform in [n_min, n_max], fractional-uniform points,
    +-1 neutral charges (the many-systems workload)."""
    rng = np.random.default_rng(seed)
    cells, pos, qs = [], [], []
    for _ in range(nsys):
        n = int(round(np.exp(rng.uniform(np.log(n_min), np.log(n_max)))))
        n += n % 2
        c = batch_cell(rng)
        frac = rng.uniform(0.0, 1.0, (n, 3))
        q = np.ones(n)
        q[: n // 2] = -1.0
        rng.shuffle(q)
        cells.append(c)
        pos.append(frac @ c.T)
        qs.append(q)
    return cells, pos, qs
