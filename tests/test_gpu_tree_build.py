"""GPU tests of the tree construction with its point steps on the device
(build_plan_device: lattice images, level-0 binning by radix sort, octant
partitions of the refinement and 2:1-balance splits, Morton order inside the
leaves).  The plan must equal the host construction's exactly: the SHA-256 of
the point order, image list, box topology and interaction lists
(pdmk_plan_digest) is compared on systems that exercise every step (deep
clustered refinement with balance splits, thin and axis-swapped triclinic
cells, many image shifts, leaves above the shared-memory Morton size).  Build
times of both forms are printed."""
import json

import numpy as np
import pytest

import periodicdmk_b200 as pd
from conftest import TRICLINIC, clustered_system, rel_l2, uniform_system

pytestmark = pytest.mark.gpu

SWAPPED = np.array([[0.8, 0.1, 0.0], [0.0, 1.3, 0.2], [0.0, 0.0, 1.0]])
THIN = np.array([[1.0, 0.2, 0.1], [0.0, 1.1, 0.3], [0.0, 0.0, 0.35]])


def _systems():
    yield "cube_1e4", uniform_system(10000, 101), 6, 50, 4
    yield "clustered_triclinic_3e4", clustered_system(30000, 102, TRICLINIC, n_clusters=6, sigma=0.01), 9, 40, 4
    yield "swapped_2e4", uniform_system(20000, 103, SWAPPED), 6, 60, 4
    yield "thin_1e4", uniform_system(10000, 104, THIN), 6, 30, 3
    yield "tiny_7", uniform_system(7, 105), 6, 300, 4
    yield "big_leaves_1e5", uniform_system(100000, 106), 3, 3000, 4  # leaves above 4096 points
    yield "clustered_cube_2e5", clustered_system(200000, 107, np.eye(3), n_clusters=16, sigma=0.005), 6, 300, 4


@pytest.mark.parametrize("case", list(range(7)))
def test_device_plan_equals_host_plan(case):
    name, (cell, pos, _), nd, npl, nz = list(_systems())[case]
    dh, th = pd.plan_digest(cell, pos, nd, npl, nz, on_device=False)
    dd, td = pd.plan_digest(cell, pos, nd, npl, nz, on_device=True)
    dd2, _ = pd.plan_digest(cell, pos, nd, npl, nz, on_device=True)
    print("BUILD " + json.dumps({"case": name, "n": len(pos), "host_ms": th, "device_ms": td}))
    assert dd == dh and dd2 == dh


def test_large_cube_build_time_and_evaluate(monkeypatch):
    cell, pos, q = uniform_system(1_000_000, 108)
    dh, th = pd.plan_digest(cell, pos, 6, 300, 4, on_device=False)
    dd, td = pd.plan_digest(cell, pos, 6, 300, 4, on_device=True)
    print("BUILD " + json.dumps({"case": "cube_1e6", "n": len(pos), "host_ms": th, "device_ms": td}))
    assert dd == dh
    # a tree built either way evaluates to the same potentials
    monkeypatch.setenv("PDMK_TREE_BUILD", "host")
    t1 = pd.PeriodicDMKTree(cell, pos, 6, 300, 4)
    u1 = t1.evaluate(q)
    t1.close()
    monkeypatch.setenv("PDMK_TREE_BUILD", "device")
    t2 = pd.PeriodicDMKTree(cell, pos, 6, 300, 4)
    u2 = t2.evaluate(q)
    t2.close()
    assert rel_l2(u2, u1) < 1e-14


def test_device_build_rejects_points_outside():
    cell, pos, _ = uniform_system(30000, 109)
    pos = pos.copy()
    pos[17] = [5.0, 0.5, 0.5]  # outside the cell's covering grid
    for dev in (False, True):
        with pytest.raises(RuntimeError, match="outside"):
            pd.plan_digest(cell, pos, 6, 300, 4, on_device=dev)


def test_points_on_cell_faces():
    # fractional coordinates exactly 0 and just below 1 on every axis: images
    # and bins at the grid edges agree between the two constructions
    rng = np.random.default_rng(110)
    frac = rng.uniform(0, 1, (40000, 3))
    frac[:5000, 0] = 0.0
    frac[5000:10000, 1] = np.nextafter(1.0, 0.0)
    frac[10000:12000, :2] = 0.0  # on an edge of the cell
    cell = TRICLINIC
    pos = frac @ cell.T
    dh, _ = pd.plan_digest(cell, pos, 6, 60, 4, on_device=False)
    dd, _ = pd.plan_digest(cell, pos, 6, 60, 4, on_device=True)
    assert dd == dh
