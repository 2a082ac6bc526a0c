"""GPU parity tests: the CUDA evaluate path (through the C ABI) against the CPU
oracle and against Ewald, on seeded inputs the oracle finishes in seconds.

Tolerances (relative L2):
  * tree part (near field + plane-wave levels - self term), FP64 path vs the
    oracle's same parts: 1e-11 (rounding only: same tree, same tables);
  * far field: NUFFT (ES kernel, tolerance eps/4) vs the oracle's exact
    reciprocal-lattice sum: 0.3 * 10^-digits of the total potential;
  * total vs oracle: 0.2 * 10^-digits (the drop-in bar is 2 * 10^-digits);
  * total vs Ewald: the reference's own bars (cpp/tests/test_periodic_dmk.cpp:42,67,
    cpp/tests/test_nonuniform.cpp:303) tightened where the method allows.
"""
import json

import numpy as np
import pytest

import oracle
import periodicdmk_b200 as pd
from conftest import TRICLINIC, clustered_system, rel_l2, uniform_system

pytestmark = pytest.mark.gpu

SYSTEMS = {
    "cube_deep": lambda: (uniform_system(3000, 21), 30),
    "triclinic_clustered": lambda: (clustered_system(3000, 22, TRICLINIC, n_clusters=4, sigma=0.02), 25),
    "cube_2e4": lambda: (uniform_system(20000, 1), 300),
}


def _tree(cell, pos, nd, npl, nz=4, precision="double"):
    return pd.PeriodicDMKTree(cell, pos, n_digits=nd, n_per_leaf=npl, nz=nz, precision=precision)


@pytest.mark.parametrize("name", ["cube_deep", "triclinic_clustered"])
@pytest.mark.parametrize("nd", [3, 6, 9, 12])
def test_parts_match_oracle(name, nd):
    (cell, pos, q), npl = SYSTEMS[name]()
    t = _tree(cell, pos, nd, npl)
    tree_part, far_part = t.evaluate_parts(q)
    ref, comp = oracle.evaluate(cell, pos, q, nd, npl, 4, components=True)
    ref_tree = comp["near"] + comp["mid"] + comp["self"]
    assert rel_l2(tree_part, ref_tree) < 1e-11
    scale = np.linalg.norm(ref)
    assert np.linalg.norm(far_part - comp["far"]) / scale < 0.3 * 10.0 ** (-nd)
    pot = t.evaluate(q)
    assert rel_l2(pot, ref) < 0.2 * 10.0 ** (-nd)
    t.close()


def test_cube_2e4_matches_oracle_and_ewald():
    # N = 20,000 cube, +-1 charges, 6 digits, npl 300: the reference's own
    # CPU-runnable case.  Against the DMK oracle (same algorithm) and against
    # an Ewald sum at every target (the physics): the drop-in bar is 2e-6.
    (cell, pos, q), npl = SYSTEMS["cube_2e4"]()
    t = _tree(cell, pos, 6, npl)
    info = t.info()
    assert info["n_boxes"] == 216 and info["n_levels"] == 1
    pot = t.evaluate(q)
    ref = oracle.evaluate(cell, pos, q, 6, npl, 4)
    assert rel_l2(pot, ref) < 2e-7
    ew = oracle.ewald_targets(cell, pos, q, np.arange(len(q)), s=6.0)
    assert rel_l2(pot, ew) < 2e-6
    assert np.abs(pot - ew).max() < 2e-6 * np.abs(ew).max()
    t.close()


@pytest.mark.parametrize("nd,tol", [(6, 1e-5), (9, 1e-8)])
def test_vs_ewald_triclinic(nd, tol):
    # cpp/tests/test_periodic_dmk.cpp:45-67 shape: triclinic cell, N=100, npl=20
    cell = np.array([[5.0, 1.0, 0.5], [0.0, 4.5, 0.8], [0.0, 0.0, 4.0]])
    rng = np.random.default_rng(77)
    frac = rng.uniform(0.01, 0.99, (100, 3))
    pos = frac @ cell.T
    q = rng.normal(size=100)
    q[0] -= q.sum()
    ref, _ = oracle.ewald_direct(cell, pos, q, 6.5)
    t = _tree(cell, pos, nd, 20)
    assert rel_l2(t.evaluate(q), ref) < tol
    t.close()


def test_repeatable_and_timed():
    (cell, pos, q), npl = SYSTEMS["cube_deep"]()
    t = _tree(cell, pos, 6, npl)
    a = t.evaluate(q)
    b = t.evaluate(q)
    c, tm = t.evaluate_timed(q)
    assert rel_l2(a, b) < 1e-12
    assert rel_l2(a, c) < 1e-10
    assert tm["dmk_ms"] > 0 and tm["direct_ms"] > 0 and tm["nufft_ms"] > 0
    # different charges give different output, linearity holds
    q2 = np.roll(q, 7)
    d = t.evaluate(q2)
    assert rel_l2(d, a) > 1e-3
    e = t.evaluate(2.0 * q - q2)
    assert rel_l2(e, 2.0 * a - d) < 1e-12
    t.close()


@pytest.mark.parametrize("nd", [6, 12])
def test_fp64_level_chunks_agree_with_one_chunk(nd, monkeypatch):
    # The FP64 pass runs level by level with a bounded transform scratch
    # (PDMK_FP64_SCRATCH_MB, read when the tree is built).  The smallest cap
    # splits every level into chunks of a few boxes; chunking only changes
    # which boxes share a launch, so the results agree to rounding (the far
    # field's atomic spreading alone makes two runs differ in the last bits).
    cell, pos, q = clustered_system(20000, 41, TRICLINIC, n_clusters=8, sigma=0.03)
    ref_tree = _tree(cell, pos, nd, 40)
    ref = ref_tree.evaluate(q)
    ref_tree.close()
    monkeypatch.setenv("PDMK_FP64_SCRATCH_MB", "16")
    t = _tree(cell, pos, nd, 40)
    assert rel_l2(t.evaluate(q), ref) < 1e-14
    t.close()
    if nd == 6:  # (the oracle takes about a minute at 12 digits on this size)
        assert rel_l2(ref, oracle.evaluate(cell, pos, q, nd, 40, 4)) < 0.2 * 10.0 ** -nd


def test_translate_image_boxes_share_expansions():
    # In a cube the box grid is aligned with the lattice, so image boxes that
    # hold exact translates of an original box's sources share its moments and
    # outgoing plane waves; triclinic images straddle boxes and none qualify.
    (cell, pos, q), npl = SYSTEMS["cube_deep"]()
    t = _tree(cell, pos, 6, npl)
    assert t.info()["translate_boxes"] > 0
    assert rel_l2(t.evaluate(q), oracle.evaluate(cell, pos, q, 6, npl, 4)) < 0.2e-6
    t.close()
    (cell, pos, q), npl = SYSTEMS["triclinic_clustered"]()
    t = _tree(cell, pos, 6, npl)
    assert t.info()["translate_boxes"] == 0
    t.close()


def test_multi_rhs_equals_single_calls():
    (cell, pos, q), npl = SYSTEMS["cube_deep"]()
    rng = np.random.default_rng(5)
    Q = rng.uniform(-1, 1, (len(q), 4))
    Q -= Q.mean(axis=0)
    t = _tree(cell, pos, 6, npl)
    P = t.evaluate_multi(Q)
    for c in range(4):
        assert rel_l2(P[:, c], t.evaluate(Q[:, c])) < 1e-12
    t.close()


def test_float_tree_close_to_double():
    (cell, pos, q), npl = SYSTEMS["cube_deep"]()
    td = _tree(cell, pos, 6, npl)
    tf = _tree(cell, pos, 6, npl, precision="float")
    a = td.evaluate(q)
    b = tf.evaluate(q)
    assert b.dtype == np.float32
    assert rel_l2(b, a) < 1e-5
    td.close()
    tf.close()


def test_single_charge_and_tiny_systems():
    # cpp/tests/test_dmk_pbc_smoke.cpp: a single charge gives a finite potential
    t = _tree(np.eye(3), np.array([[0.3, 0.4, 0.5]]), 6, 300)
    v = t.evaluate(np.array([1.0]))
    assert np.all(np.isfinite(v))
    ref = oracle.evaluate(np.eye(3), np.array([[0.3, 0.4, 0.5]]), np.array([1.0]), 6, 300, 4)
    assert abs(v[0] - ref[0]) < 0.2e-6 * max(1.0, abs(ref[0]))
    t.close()
    cell, pos, q = uniform_system(2, 3)
    t = _tree(cell, pos, 9, 1)
    assert rel_l2(t.evaluate(q), oracle.evaluate(cell, pos, q, 9, 1, 4)) < 1e-9
    t.close()


def test_zero_charges_give_zero():
    cell, pos, q = uniform_system(500, 4)
    t = _tree(cell, pos, 6, 30)
    assert np.all(t.evaluate(np.zeros_like(q)) == 0.0)
    t.close()


def test_errors_on_device_tree():
    cell, pos, q = uniform_system(100, 4)
    t = _tree(cell, pos, 6, 30)
    with pytest.raises(ValueError):
        t.evaluate(q[:-1])
    t.close()
    with pytest.raises(RuntimeError, match="bloch|outside|n_digits|nz"):
        _tree(cell, pos + 5.0, 6, 30)


@pytest.mark.parametrize("nd", [9, 12])
def test_fp64_translations_on_dmma(nd, monkeypatch):
    # PDMK_FP64_DMMA=1 (read when the tree is built) runs the child <-> parent
    # translations on mma.sync.m8n8k4.f64 (the default at 9 digits), 0 on the
    # CUDA cores (the default at 12); same arithmetic up to the order of the
    # FP64 sums, so the two agree to rounding
    cell, pos, q = clustered_system(20000, 41, TRICLINIC, n_clusters=8, sigma=0.03)
    monkeypatch.setenv("PDMK_FP64_DMMA", "0")
    ref_tree = _tree(cell, pos, nd, 40)
    ref = ref_tree.evaluate(q)
    ref_tree.close()
    monkeypatch.setenv("PDMK_FP64_DMMA", "1")
    t = _tree(cell, pos, nd, 40)
    assert rel_l2(t.evaluate(q), ref) < 1e-13
    t.close()


@pytest.mark.parametrize("nd", [9, 12])
def test_fp64_moments_on_dmma(nd, monkeypatch):
    # PDMK_MOMENTS_DMMA=1 (read when the tree is built) forms the proxy moments
    # of the orders p = 28, 38 on mma.sync.m8n8k4.f64: the same sums in another
    # order, so the potentials agree with the CUDA-core kernel to rounding
    cell, pos, q = clustered_system(20000, 42, TRICLINIC, n_clusters=8, sigma=0.03)
    monkeypatch.setenv("PDMK_MOMENTS_DMMA", "0")
    ref_tree = _tree(cell, pos, nd, 40)
    ref = ref_tree.evaluate(q)
    ref_tree.close()
    monkeypatch.setenv("PDMK_MOMENTS_DMMA", "1")
    t = _tree(cell, pos, nd, 40)
    assert rel_l2(t.evaluate(q), ref) < 1e-13
    t.close()


def test_float_tree_vs_oracle():
    # the float tree (mixed precision, one RHS) against the FP64 oracle at 6
    # digits: the north-star bar for the mixed path, 1e-6 relative L2
    (cell, pos, q), npl = SYSTEMS["cube_deep"]()
    tf = _tree(cell, pos, 6, npl, precision="float")
    b = tf.evaluate(q)
    tf.close()
    ref = oracle.evaluate(cell, pos, q, 6, npl, 4)
    e = rel_l2(b, ref)
    print("PARITY " + json.dumps({"case": "float tree, one RHS, 6 digits", "rel_l2_vs_oracle": e}))
    assert e < 1e-6
