"""Host-side checks of bench.py's workload generators (no GPU)."""
import numpy as np

import bench


def test_clustered_system_matches_its_description():
    cell, pos, q = bench.clustered_system(4000, seed=3)
    assert pos.shape == (4000, 3) and q.shape == (4000,)
    assert np.allclose(cell[:, 0], [1.0, 0.0, 0.0]) and np.allclose(cell[:, 1], [0.3, 0.9, 0.0])
    assert np.allclose(cell[:, 2], [0.2, 0.25, 0.85])
    assert set(np.unique(q)) == {-1.0, 1.0} and q.sum() == 0.0
    frac = pos @ np.linalg.inv(cell).T
    assert np.all(frac >= 0.0) and np.all(frac < 1.0)
    # the clustered half is far more concentrated than the uniform half
    nn_u = np.sort(np.linalg.norm(pos[:200, None] - pos[None, :2000], axis=2), axis=1)[:, 1].mean()
    nn_c = np.sort(np.linalg.norm(pos[2000:2200, None] - pos[None, 2000:], axis=2), axis=1)[:, 1].mean()
    assert nn_c < 0.5 * nn_u
    cell2, pos2, q2 = bench.clustered_system(4000, seed=3)
    assert np.array_equal(pos, pos2) and np.array_equal(q, q2)


def test_host_binding_helpers_without_a_gpu():
    """Without a usable GPU or NVML the bench keeps the process affinity and
    still names a device for nvidia-smi (its index)."""
    import os

    import torch

    if torch.cuda.is_available():
        return
    before = os.sched_getaffinity(0)
    assert bench.bind_host_to_gpu(0) is None
    assert os.sched_getaffinity(0) == before
    assert bench.smi_id(0) == "0"
