"""CPU tests: pin the oracle and the product's host math against the reference's
golden vectors and independent physics (no GPU).

Golden sources:
  tests/golden/pswf.json, legendre.json, images.json  -- generated from the
      reference's own prolate.cpp / legeexps.cpp / pbc.hpp / image_layout.hpp
      by tests/golden/make_golden.py
  NaCl Madelung constant 1.7475645946331822 (cpp/tests/test_ewald_nufft.cpp:69)
  DMK vs Ewald tolerances (cpp/tests/test_periodic_dmk.cpp:42,67: 1e-4 at 6 digits;
      cpp/tests/test_nonuniform.cpp:303: 1e-7 at 9 digits)
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from conftest import TRICLINIC, batch_systems, clustered_system, rel_l2, uniform_system

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


@pytest.mark.parametrize("case", range(4))
def test_pswf_matches_reference(case):
    g = _load("pswf.json")[case]
    psi, m = oracle.pswf(g["beta"], np.array(g["x"]))
    np.testing.assert_allclose(psi, g["psi"], rtol=0, atol=1e-13)
    assert abs(m[0] / g["c0"] - 1) < 1e-12
    assert abs(m[2] / g["c2"] - 1) < 1e-12
    assert abs(m[3] / g["c4"] - 1) < 1e-12


def test_pswf_known_values():
    # psi_0(0) and c0 of the four digit brackets, from the reference's prolate.cpp
    table = [(7.2462000846862793, 1.2139916469720284, 0.56522128362727631),
             (13.739999771118164, 1.4355921697404228, 0.4853976357105198),
             (20.736000061035156, 1.5952924421089012, 0.43907403292843861),
             (27.870000839233398, 1.7198365570788461, 0.40829928909079977)]
    for beta, psi0, c0 in table:
        psi, m = oracle.pswf(beta, np.array([0.0]))
        assert abs(psi[0] / psi0 - 1) < 1e-14
        assert abs(m[0] / c0 - 1) < 1e-12


@pytest.mark.parametrize("n", [100, 200])
def test_gauss_legendre_matches_reference(n):
    g = _load("legendre.json")[str(n)]
    x, w = oracle.legendre(n)
    np.testing.assert_allclose(x, g["x"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(w, g["w"], rtol=1e-12, atol=0)


def _golden_system(name):
    if name == "cube_n20000_seed1":
        return uniform_system(20000, 1)
    if name == "cube_n3000_seed2_nz7":
        return uniform_system(3000, 2)
    if name == "triclinic_n4000_seed3":
        return uniform_system(4000, 3, TRICLINIC)
    if name == "triclinic_clustered_n4000_seed4":
        return clustered_system(4000, 4, TRICLINIC)
    if name == "swapped_axes_n2000_seed5":
        return uniform_system(2000, 5, np.array([[0.8, 0.1, 0.0], [0, 1.3, 0.2], [0, 0, 1.0]]))
    raise KeyError(name)


@pytest.mark.parametrize("case", range(5))
def test_geometry_and_images_match_reference(case):
    g = _load("images.json")[case]
    cell, pos, _ = _golden_system(g["name"])
    umat, qmat, mg, xg, rc, idx = oracle.plan_images(cell, pos, g["nz"])
    np.testing.assert_allclose(umat, g["umat"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(qmat, g["qmat"], rtol=0, atol=1e-15)
    assert list(mg) == g["mgrid"]
    np.testing.assert_allclose(xg, g["xgrid0"], rtol=0, atol=1e-15)
    assert rc == g["rc"]
    assert len(idx) == g["n_images"]
    assert list(idx[:64]) == g["img_idx_head"]
    assert hashlib.sha256(idx.astype("<i4").tobytes()).hexdigest() == g["img_idx_sha256"]


def test_madelung_constant():
    pos = np.array([[0, 0, 0], [.5, .5, 0], [.5, 0, .5], [0, .5, .5], [.5, 0, 0], [0, .5, 0], [0, 0, .5],
                    [.5, .5, .5]])
    q = np.array([1, 1, 1, 1, -1, -1, -1, -1.0])
    _, e = oracle.ewald_direct(np.eye(3), pos, q, 5.5)
    assert abs(-e / 8.0 - 1.7475645946331822) < 1e-8


def test_oracle_dmk_madelung():
    # The DMK oracle on the NaCl cell reproduces the Madelung energy.
    pos = np.array([[0, 0, 0], [.5, .5, 0], [.5, 0, .5], [0, .5, .5], [.5, 0, 0], [0, .5, 0], [0, 0, .5],
                    [.5, .5, .5]]) + 0.01
    q = np.array([1, 1, 1, 1, -1, -1, -1, -1.0])
    pot = oracle.evaluate(np.eye(3), pos, q, n_digits=9, n_per_leaf=20, nz=4)
    assert abs(-0.5 * np.dot(q, pot) / 8.0 - 1.7475645946331822) < 1e-7


@pytest.mark.parametrize("nd,tol", [(3, 3e-3), (6, 1e-5), (9, 1e-8), (12, 1e-10)])
def test_oracle_vs_ewald_cubic(nd, tol):
    # cpp/tests/test_periodic_dmk.cpp:20-43 shape: cubic L=3, N=200, npl=20, nz=4
    rng = np.random.default_rng(42)
    L = 3.0
    pos = rng.uniform(0.03 * L, 0.97 * L, (200, 3))
    q = rng.normal(size=200)
    q[0] -= q.sum()
    ref, _ = oracle.ewald_direct(np.eye(3) * L, pos, q, 6.0)
    pot = oracle.evaluate(np.eye(3) * L, pos, q, nd, 20, 4)
    assert rel_l2(pot, ref) < tol


@pytest.mark.parametrize("nd,tol", [(6, 1e-5), (9, 5e-8)])
def test_oracle_vs_ewald_triclinic_deep(nd, tol):
    cell, pos, q = clustered_system(1500, 11, TRICLINIC, n_clusters=3, sigma=0.02)
    ref, _ = oracle.ewald_direct(cell, pos, q, 6.5)
    pot = oracle.evaluate(cell, pos, q, nd, 15, 4)
    assert rel_l2(pot, ref) < tol
    assert oracle.plan_stats(cell, pos, nd, 15, 4)["nlevels"] >= 3


def test_oracle_nz_independence():
    cell, pos, q = uniform_system(600, 5)
    a = oracle.evaluate(cell, pos, q, 9, 20, 3)
    b = oracle.evaluate(cell, pos, q, 9, 20, 5)
    assert rel_l2(a, b) < 1e-7


def test_oracle_linearity_and_charge_flip():
    cell, pos, q = uniform_system(500, 8)
    rng = np.random.default_rng(3)
    q2 = rng.uniform(-1, 1, 500)
    q2 -= q2.mean()
    a = oracle.evaluate(cell, pos, q, 6, 20, 4)
    b = oracle.evaluate(cell, pos, q2, 6, 20, 4)
    c = oracle.evaluate(cell, pos, 2.0 * q - 0.5 * q2, 6, 20, 4)
    assert rel_l2(c, 2.0 * a - 0.5 * b) < 1e-12
    assert rel_l2(oracle.evaluate(cell, pos, -q, 6, 20, 4), -a) < 1e-14


def test_plan_sizes_uniform_cube():
    # N=20000 uniform cube, 6 digits, npl 300, nz 4: one level of 6^3 boxes,
    # 64 inner leaves, 18^3 far-field modes.
    cell, pos, _ = uniform_system(20000, 1)
    st = oracle.plan_stats(cell, pos, 6, 300, 4)
    assert st["nboxes"] == 216 and st["nlevels"] == 1
    assert st["n_target_leaves"] == 64
    assert (st["ms"], st["mt"], st["mu"]) == (18, 18, 18)
    assert st["n_all"] == 20000 + _load("images.json")[0]["n_images"]


def test_ewald_targets_matches_direct_ewald():
    # The sampled-target Ewald (cell list + separable reciprocal sum), used as
    # the physics check at full sizes, equals the all-pairs Ewald sum on a
    # small clustered triclinic system for any splitting parameter alpha.
    cell, pos, q = clustered_system(600, 5, TRICLINIC, n_clusters=3, sigma=0.05)
    ref, _ = oracle.ewald_direct(cell, pos, q, 6.5)
    for alpha in (0.0, 5.0, 12.0):
        v = oracle.ewald_targets(cell, pos, q, np.arange(len(q)), s=6.5, alpha=alpha)
        assert rel_l2(v, ref) < 1e-14
    idx = np.array([3, 100, 599, 250])
    assert rel_l2(oracle.ewald_targets(cell, pos, q, idx, s=6.5), ref[idx]) < 1e-14


def test_oracle_multi_equals_single_columns():
    cell, pos, _ = uniform_system(1500, 8)
    rng = np.random.default_rng(3)
    Q = rng.uniform(-1, 1, (1500, 3))
    Q -= Q.mean(axis=0)
    P = oracle.evaluate_multi(cell, pos, Q, 6, 40, 4)
    for c in range(3):
        assert rel_l2(P[:, c], oracle.evaluate(cell, pos, Q[:, c], 6, 40, 4)) < 1e-14


def _assert_same_tree(r):
    bad = {k: v for k, v in r.items() if k.endswith("_mismatch") and v != 0}
    assert not bad, (bad, r)


@pytest.mark.parametrize("case", range(5))
@pytest.mark.parametrize("npl", [20, 300])
def test_independent_tree_matches_plan_golden_systems(case, npl):
    # The oracle's own tree builder (oracle/oracle_tree.cpp: integer box keys,
    # per-point descent, 2:1 balance as a fixed point) and the product's host
    # plan give the same boxes, leaf point sets, plane-wave flags, near lists
    # with their cutoffs, moment work and direct work on the golden systems.
    g = _load("images.json")[case]
    cell, pos, _ = _golden_system(g["name"])
    r = oracle.tree_compare(cell, pos, 6, npl, g["nz"])
    _assert_same_tree(r)
    assert r["boxes"] >= r["boxes_l0"] > 0


def test_independent_tree_matches_plan_clustered_triclinic():
    # the clustered triclinic workload's shape (half the points in 64 Gaussian
    # clusters of sigma 0.01) at 2e5 points: deep, 2:1-balanced trees
    cell, pos, _ = clustered_system(200000, 3, TRICLINIC, n_clusters=64, sigma=0.01)
    r = oracle.tree_compare(cell, pos, 9, 300, 4)
    _assert_same_tree(r)
    assert r["levels"] >= 4


def test_independent_tree_matches_plan_batch_cells():
    # random triclinic cells of the many-systems workload (axis sorting in the
    # lattice QR, oblique images)
    cells, pos, _ = batch_systems(6, 17, n_min=1000, n_max=20000)
    for c, p in zip(cells, pos):
        _assert_same_tree(oracle.tree_compare(c, p, 6, 300, 4))


def test_ewald_gradient_matches_finite_differences():
    # d phi_t / d x_t of the sampled-target Ewald sum against central
    # differences (moving a point moves its charge: its own images and the self
    # term do not depend on its position, so the derivative is the field of the
    # other charges)
    cell, pos, q = clustered_system(400, 9, TRICLINIC, n_clusters=3, sigma=0.05)
    idx = np.array([0, 57, 203, 399])
    _, g = oracle.ewald_targets_grad(cell, pos, q, idx, s=6.5)
    h = 1e-5
    for row, t in enumerate(idx):
        for d in range(3):
            pp, pm = pos.copy(), pos.copy()
            pp[t, d] += h
            pm[t, d] -= h
            fd = (oracle.ewald_targets(cell, pp, q, [t], s=6.5)[0] - oracle.ewald_targets(cell, pm, q, [t], s=6.5)[0]) / (2 * h)
            assert abs(fd - g[row, d]) < 1e-6 * max(1.0, np.abs(g[row]).max()), (t, d, fd, g[row, d])
    # potentials unchanged by the gradient pass
    v, _ = oracle.ewald_targets_grad(cell, pos, q, idx, s=6.5)
    assert rel_l2(v, oracle.ewald_targets(cell, pos, q, idx, s=6.5)) < 1e-15


def test_quasi_periodic_ewald_oracle():
    # Bloch vector 0 reproduces the periodic Ewald sum; for a nonzero Bloch
    # vector the result does not depend on the splitting parameter alpha
    cell, pos, q = clustered_system(500, 5, TRICLINIC, n_clusters=3, sigma=0.05)
    idx = np.arange(len(q))
    ref = oracle.ewald_targets(cell, pos, q, idx, s=6.5)
    z = oracle.ewald_targets_qp(cell, pos, q, idx, [0.0, 0.0, 0.0], s=6.5)
    assert rel_l2(z.real, ref) < 1e-14 and np.abs(z.imag).max() < 1e-13 * np.abs(ref).max()
    b = np.array([0.7, -1.1, 2.3])
    z1 = oracle.ewald_targets_qp(cell, pos, q, idx, b, s=6.5)
    z2 = oracle.ewald_targets_qp(cell, pos, q, idx, b, s=6.5, alpha=9.0)
    assert np.linalg.norm(z1 - z2) / np.linalg.norm(z1) < 1e-13
