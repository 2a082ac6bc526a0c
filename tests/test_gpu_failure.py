"""Failure detection of the tensor-core pipeline, exercised without a GPU fault.

The tensor-core kernels wait on their MMA-completion barriers with a bound;
when a wait runs out, the CTA stops issuing, waits (bounded) for its own MMAs
in flight, frees its tensor memory and sets a device error word, which the
host turns into -2 at the C ABI.  The test hook PDMK_TEST_WITHHOLD_NEAR_CHUNK
makes the first target tile of the near-field kernel skip one chunk's MMAs and
commits -- a barrier that nothing completes -- with a ~10 ms wait budget; the
call must return -2 with the timeout message, and the next evaluate on the
same tree must succeed and match the one before."""
import ctypes

import numpy as np
import pytest

import periodicdmk_b200 as pd
from conftest import rel_l2, uniform_system

pytestmark = pytest.mark.gpu


def test_near_field_wait_timeout_returns_minus_2_and_tree_recovers(monkeypatch):
    import torch

    monkeypatch.delenv("PDMK_TEST_WITHHOLD_NEAR_CHUNK", raising=False)
    cell, pos, _ = uniform_system(8000, 60)
    rng = np.random.default_rng(9)
    Q = rng.uniform(-1.0, 1.0, (len(pos), 16))
    Q -= Q.mean(axis=0)
    t = pd.PeriodicDMKTree(cell, pos, 6, 100, 4, precision="float")
    dev = torch.device("cuda", torch.cuda.current_device())
    q_d = torch.from_numpy(np.ascontiguousarray(Q.T)).to(dev)
    p_d = torch.empty_like(q_d)
    lib = pd.library()

    def call():
        torch.cuda.synchronize()
        return lib.pdmk_evaluate_multi_device_float(t._h, 16, ctypes.c_void_p(q_d.data_ptr()),
                                                    ctypes.c_void_p(p_d.data_ptr()))

    assert call() == 0
    ref = p_d.cpu().numpy()
    monkeypatch.setenv("PDMK_TEST_WITHHOLD_NEAR_CHUNK", "0")
    assert call() == -2
    assert "timed out" in pd._last_error()
    monkeypatch.delenv("PDMK_TEST_WITHHOLD_NEAR_CHUNK")
    assert call() == 0, pd._last_error()
    again = p_d.cpu().numpy()
    assert np.all(np.isfinite(again))
    assert rel_l2(again, ref) < 1e-12
    t.close()
