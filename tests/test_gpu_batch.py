"""GPU tests of the batch entry points (pdmk_batch_*): many independent
systems built together and evaluated concurrently, each checked against the
single-system tree of the same precision (same arithmetic) and the mixed
precision batch against FP64 trees (1e-6 rel L2 per system)."""
import numpy as np
import pytest

import periodicdmk_b200 as pd
from conftest import batch_systems, rel_l2

pytestmark = pytest.mark.gpu


def test_mixed_batch_matches_single_trees():
    cells, pos, qs = batch_systems(6, 51, n_min=1000, n_max=20000)
    b = pd.PeriodicDMKBatch(cells, pos, n_digits=6, n_per_leaf=300, nz=4)
    info = b.info()
    assert info["n_systems"] == 6 and info["float_trees"] and info["n_points"] == sum(len(q) for q in qs)
    out = b.evaluate(qs)
    out32 = b.evaluate(qs, out_dtype=np.float32)
    for c, p, q, u, u32 in zip(cells, pos, qs, out, out32):
        tf = pd.PeriodicDMKTree(c, p, 6, 300, 4, precision="float")
        td = pd.PeriodicDMKTree(c, p, 6, 300, 4)
        assert rel_l2(u, tf.evaluate(q)) < 1e-7  # float trees return float32 potentials
        assert rel_l2(u, td.evaluate(q)) < 1e-6
        assert u32.dtype == np.float32 and rel_l2(u32, u) < 1e-7
        tf.close()
        td.close()
    # repeat: same result
    again = b.evaluate(qs)
    for u, v in zip(out, again):
        assert rel_l2(v, u) < 1e-12
    # concatenated charges and a preallocated output (written in place)
    flat = np.concatenate(qs)
    buf = np.full(flat.shape[0], np.nan)
    views = b.evaluate(flat, out=buf)
    assert np.all(np.isfinite(buf))
    for u, v in zip(out, views):
        assert rel_l2(v, u) < 1e-12
    # page-locked host buffers are copied by DMA directly (no staging)
    import torch

    qp = torch.from_numpy(flat).pin_memory()
    pp = torch.empty(flat.shape[0], dtype=torch.float64).pin_memory()
    b.evaluate(qp.numpy(), out=pp.numpy())
    for i, u in enumerate(out):
        assert rel_l2(pp.numpy()[b.offsets[i]:b.offsets[i + 1]], u) < 1e-12
    with pytest.raises(ValueError):
        b.evaluate(flat, out=np.empty(flat.shape[0], dtype=np.float32))
    b.close()


def test_double_batch_matches_single_trees():
    cells, pos, qs = batch_systems(4, 52, n_min=1000, n_max=8000)
    b = pd.PeriodicDMKBatch(cells, pos, n_digits=9, n_per_leaf=200, nz=4)
    assert not b.info()["float_trees"]
    out = b.evaluate(qs)
    for c, p, q, u in zip(cells, pos, qs, out):
        td = pd.PeriodicDMKTree(c, p, 9, 200, 4)
        assert rel_l2(u, td.evaluate(q)) < 1e-12
        td.close()
    b.close()
    b2 = pd.PeriodicDMKBatch(cells, pos, n_digits=6, n_per_leaf=300, nz=4, precision="double")
    assert not b2.info()["float_trees"]
    out2 = b2.evaluate(qs)
    for c, p, q, u in zip(cells, pos, qs, out2):
        td = pd.PeriodicDMKTree(c, p, 6, 300, 4)
        assert rel_l2(u, td.evaluate(q)) < 1e-12
        td.close()
    b2.close()


def test_batch_errors():
    cells, pos, qs = batch_systems(2, 53, n_min=1000, n_max=2000)
    b = pd.PeriodicDMKBatch(cells, pos)
    with pytest.raises(ValueError):
        b.evaluate([qs[0]])
    b.close()
    lib = pd.library()
    assert lib.pdmk_batch_evaluate(None, None, None) == -1
