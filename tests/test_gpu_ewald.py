"""GPU tests of the Ewald summation entry point (pdmk_ewald_nufft; cell-list
real-space sum and NUFFT reciprocal sum on the device), as the reference tests
its ewald_nufft (cpp/tests/test_ewald_nufft.cpp): the NaCl Madelung constant
to 1e-8 and agreement with a direct Ewald sum, here the oracle's
(oracle.ewald_direct on small systems, oracle.ewald_targets at sampled
targets of larger ones; both CPU).  It then serves as the large-N reference:
at N = 1e6 it agrees with the 12-digit DMK evaluate, and its potentials are
stored in and read back from a campaign reference file."""
import json
import time

import numpy as np
import pytest

import oracle
import periodicdmk_b200 as pd
from conftest import TRICLINIC, clustered_system, rel_l2, uniform_system
from periodicdmk_b200 import campaign

pytestmark = pytest.mark.gpu

NACL = np.array([[0, 0, 0], [.5, .5, 0], [.5, 0, .5], [0, .5, .5], [.5, 0, 0], [0, .5, 0], [0, 0, .5], [.5, .5, .5]])


def test_madelung_nacl():
    q = np.array([1, 1, 1, 1, -1, -1, -1, -1.0])
    pot, e = pd.ewald(np.eye(3), NACL, q, 5.5)
    assert abs(-e / 8 - 1.7475645946331822) < 1e-8
    # every ion sees the Madelung potential -/+ 2 M (unit spacing 1/2)
    assert np.abs(np.abs(pot) - 2 * 1.7475645946331822).max() < 1e-8


def test_small_triclinic_matches_direct():
    cell, pos, q = uniform_system(64, 3, TRICLINIC, charges="uniform")
    a, ea = pd.ewald(cell, pos, q, 5.5)
    b, eb = oracle.ewald_direct(cell, pos, q, 5.5)
    assert rel_l2(a, b) < 1e-10
    assert abs(ea - eb) < 1e-10 * abs(eb)
    assert abs(ea - 0.5 * np.dot(q, a)) < 1e-12 * abs(ea)  # neutral: no charged-system term


def test_thin_cell_and_positions_outside():
    # a cell thinner than the real-space cutoff along one axis (several image
    # layers in the bin stencil) and positions given outside the cell
    cell = np.array([[1.0, 0.2, 0.1], [0.0, 1.1, 0.3], [0.0, 0.0, 0.12]])
    rng = np.random.default_rng(5)
    frac = rng.uniform(0, 1, (300, 3))
    q = rng.choice([-1.0, 1.0], 300)
    q -= q.mean()
    pos = frac @ cell.T
    shifted = pos + np.outer(rng.integers(-2, 3, 300), cell[:, 0]) + np.outer(rng.integers(-1, 2, 300), cell[:, 2])
    a, _ = pd.ewald(cell, pos, q, 5.0)
    b, _ = pd.ewald(cell, shifted, q, 5.0)
    ref = oracle.ewald_targets(cell, pos, q, np.arange(300), s=6.0)
    assert rel_l2(a, ref) < 1e-9 and rel_l2(b, ref) < 1e-9


@pytest.mark.parametrize("system", ["cube", "clustered_triclinic"])
def test_sampled_targets_vs_oracle(system):
    if system == "cube":
        cell, pos, q = uniform_system(20000, 91)
    else:
        cell, pos, q = clustered_system(20000, 92, TRICLINIC, n_clusters=8, sigma=0.02)
    pot, _ = pd.ewald(cell, pos, q, 4.8)
    idx = np.random.default_rng(1).choice(len(q), 300, replace=False)
    ref = oracle.ewald_targets(cell, pos, q, idx, s=6.5)
    e = rel_l2(pot[idx], ref)
    print("PARITY " + json.dumps({"case": "GPU Ewald %s N=2e4, s=4.8" % system, "rel_l2_vs_oracle_300": e}))
    assert e < 1e-9


def test_large_n_reference_and_campaign_file(tmp_path):
    cell, pos, q = uniform_system(1_000_000, 93)
    t0 = time.perf_counter()
    pot, e = pd.ewald(cell, pos, q, 4.8)
    t_ewald = time.perf_counter() - t0
    idx = np.random.default_rng(2).choice(len(q), 128, replace=False)
    ref = oracle.ewald_targets(cell, pos, q, idx, s=6.5)
    tree = pd.PeriodicDMKTree(cell, pos, 12, 300, 4)
    dmk = tree.evaluate(q)
    tree.close()
    e_or, e_dmk = rel_l2(pot[idx], ref), rel_l2(pot, dmk)
    print("PARITY " + json.dumps({"case": "GPU Ewald N=1e6 cube, s=4.8", "seconds": t_ewald,
                                  "rel_l2_vs_oracle_128": e_or, "rel_l2_vs_dmk_12_digits": e_dmk}))
    assert e_or < 1e-9 and e_dmk < 1e-9
    # store the reference at 1000 sampled points and check the 6-digit DMK against it
    sample = np.random.default_rng(3).choice(len(q), campaign.DEFAULT_M, replace=False)
    path = str(tmp_path / "cube1e6.pdmc")
    campaign.write_ref(path, cell, pos, q, sample, pot[sample], config_id=2, digits=12, prec=1, seed=93)
    d = campaign.read_ref(path)
    assert d["N"] == len(q) and d["M"] == campaign.DEFAULT_M
    t6 = pd.PeriodicDMKTree(d["cell"], d["positions"], 6, 300, 4)
    u6 = t6.evaluate(d["charges"])
    t6.close()
    assert rel_l2(u6[d["ref_idx"]], d["ref_u"]) < 2e-6


def test_errors():
    with pytest.raises(RuntimeError, match="degenerate"):
        pd.ewald(np.zeros((3, 3)), NACL, np.ones(8), 5.0)
    with pytest.raises(RuntimeError, match="s must be positive"):
        pd.ewald(np.eye(3), NACL, np.ones(8), -1.0)
