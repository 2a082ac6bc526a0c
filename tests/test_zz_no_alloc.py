"""GPU test of the evaluate entry point that allocates no device memory.

It is for callers that cannot allocate device memory while running (their own
allocator owns the GPU pool, or they cannot take cudaMalloc's device-wide
synchronisation in a time-step loop).  The test calls it through the C ABI on
device buffers the test owns, twice in a row (the static scratch array keeps
the previous call's contents), and checks each result against the regular
device evaluate; around the second call the device's free memory must not
change.  This file is collected last so a failure here never hides another
test's result.
"""
import ctypes

import numpy as np
import pytest

import periodicdmk_b200 as pd
from conftest import TRICLINIC, clustered_system, rel_l2, uniform_system

pytestmark = pytest.mark.gpu


# The 12-digit case needs 84,700 complex plane-wave values (1.36 MB) of
# transform scratch per box, so the 32 MiB array holds 24 boxes at a time and
# its levels (hundreds of boxes) run in many chunks.
@pytest.mark.parametrize("system,n,nd,npl", [("cube", 3000, 6, 30), ("triclinic", 3000, 9, 25),
                                             ("triclinic", 20000, 12, 40)])
def test_noalloc_matches_regular_evaluate_twice(system, n, nd, npl):
    import torch

    if system == "cube":
        cell, pos, q = uniform_system(n, 31)
    else:
        cell, pos, q = clustered_system(n, 32, TRICLINIC, n_clusters=4, sigma=0.02)
    lib = pd.library()
    t = pd.PeriodicDMKTree(cell, pos, n_digits=nd, n_per_leaf=npl, nz=4)
    dev = torch.device("cuda", torch.cuda.current_device())
    q_d = torch.from_numpy(q).to(dev)
    ref_d = torch.empty(len(q), dtype=torch.float64, device=dev)
    out_d = torch.full((len(q),), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    assert lib.pdmk_evaluate_device_double(t._h, ctypes.c_void_p(q_d.data_ptr()),
                                           ctypes.c_void_p(ref_d.data_ptr())) == 0
    ref = ref_d.cpu().numpy()
    for call in range(2):
        out_d.fill_(float("nan"))
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = lib.pdmk_evaluate_device_noalloc_double(t._h, ctypes.c_void_p(q_d.data_ptr()),
                                                     ctypes.c_void_p(out_d.data_ptr()))
        assert rc == 0, pd._last_error()
        free_after = torch.cuda.mem_get_info()[0]
        if call == 1:
            assert free_after == free_before
        out = out_d.cpu().numpy()
        assert np.all(np.isfinite(out))
        assert rel_l2(out, ref) < 1e-13
    t.close()


def test_noalloc_null_handle():
    lib = pd.library()
    assert lib.pdmk_evaluate_device_noalloc_double(None, None, None) == -1
    assert "null handle" in pd._last_error()
