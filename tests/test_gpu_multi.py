"""GPU tests of the multi-RHS evaluate (k charge vectors on one tree) and of the
mixed-precision path, through the C ABI.

Tolerances (relative L2, per charge vector):
  * plain FP64 multi-RHS vs single-RHS FP64 evaluates: 1e-12 (same arithmetic);
  * mixed precision vs the FP64 path: 1e-6 at 6 digits (the accuracy target of
    the batched mode), 2e-4 at 3 digits; both also vs the CPU oracle;
  * n_digits > 6 with mixed requested: the FP64 path runs (1e-12 vs FP64).
Blocks of 16 or more RHS form the proxy moments on the tensor cores (TF32
hi/lo split); blocks of fewer RHS use the CUDA-core kernel.  Both are held to
the same tolerances.
"""
import ctypes

import json

import numpy as np
import pytest

import oracle
import periodicdmk_b200 as pd
from conftest import TRICLINIC, clustered_system, rel_l2, uniform_system

pytestmark = pytest.mark.gpu


def _charges(n, k, seed):
    rng = np.random.default_rng(seed)
    Q = rng.uniform(-1.0, 1.0, (n, k))
    Q -= Q.mean(axis=0)
    return Q


def _multi_device(tree, Q, mixed):
    import torch

    dev = torch.device("cuda", torch.cuda.current_device())
    q_d = torch.from_numpy(np.ascontiguousarray(Q.T)).to(dev)  # column-major N x k
    p_d = torch.empty_like(q_d)
    torch.cuda.synchronize()
    tree.evaluate_multi_device(Q.shape[1], q_d.data_ptr(), p_d.data_ptr(), mixed=mixed)
    return p_d.cpu().numpy().T


@pytest.mark.parametrize("system", ["cube", "triclinic"])
def test_fp64_multi_equals_single(system):
    if system == "cube":
        cell, pos, _ = uniform_system(3000, 41)
    else:
        cell, pos, _ = clustered_system(3000, 42, TRICLINIC, n_clusters=4, sigma=0.02)
    Q = _charges(len(pos), 5, 1)
    t = pd.PeriodicDMKTree(cell, pos, 6, 30, 4)
    P = _multi_device(t, Q, mixed=False)
    for c in range(5):
        assert rel_l2(P[:, c], t.evaluate(Q[:, c])) < 1e-12
    # host-buffer path, same numbers
    P2 = t.evaluate_multi(Q)
    assert rel_l2(P2, P) < 1e-14
    t.close()


@pytest.mark.parametrize("nd,tol", [(6, 1e-6), (3, 2e-4)])
@pytest.mark.parametrize("system", ["cube", "triclinic"])
def test_mixed_multi_accuracy(system, nd, tol):
    if system == "cube":
        cell, pos, _ = uniform_system(4000, 43)
        npl = 40
    else:
        cell, pos, _ = clustered_system(4000, 44, TRICLINIC, n_clusters=4, sigma=0.02)
        npl = 30
    Q = _charges(len(pos), 8, 2)
    t = pd.PeriodicDMKTree(cell, pos, nd, npl, 4)
    Pm = _multi_device(t, Q, mixed=True)
    Pd = _multi_device(t, Q, mixed=False)
    for c in range(8):
        assert rel_l2(Pm[:, c], Pd[:, c]) < tol, c
    ref = oracle.evaluate(cell, pos, Q[:, 0], nd, npl, 4)
    assert rel_l2(Pm[:, 0], ref) < tol + 0.2 * 10.0 ** (-nd)
    t.close()


def test_mixed_request_above_six_digits_runs_fp64():
    cell, pos, _ = uniform_system(2000, 45)
    Q = _charges(len(pos), 3, 3)
    t = pd.PeriodicDMKTree(cell, pos, 9, 30, 4)
    Pm = _multi_device(t, Q, mixed=True)
    Pd = _multi_device(t, Q, mixed=False)
    assert rel_l2(Pm, Pd) < 1e-13
    t.close()


def test_rhs_blocks_tail():
    # k = 70 > the 64-RHS block: two blocks (64 + 6)
    cell, pos, _ = uniform_system(1500, 46)
    Q = _charges(len(pos), 70, 4)
    t = pd.PeriodicDMKTree(cell, pos, 6, 40, 4)
    P = t.evaluate_multi(Q)
    for c in (0, 63, 64, 69):
        assert rel_l2(P[:, c], t.evaluate(Q[:, c])) < 1e-12
    t.close()


def test_float_tree_mixed_path():
    cell, pos, q = uniform_system(4000, 47, charges="uniform")
    td = pd.PeriodicDMKTree(cell, pos, 6, 40, 4)
    tf = pd.PeriodicDMKTree(cell, pos, 6, 40, 4, precision="float")
    a = td.evaluate(q)
    b = tf.evaluate(q)
    assert b.dtype == np.float32
    assert rel_l2(b, a) < 1e-6
    c, tm = tf.evaluate_timed(q)
    assert rel_l2(c, b) < 1e-7 and tm["direct_ms"] > 0
    Q = _charges(len(q), 4, 5)
    F = tf.evaluate_multi(Q)
    assert F.dtype == np.float32
    for j in range(4):
        assert rel_l2(F[:, j], td.evaluate(Q[:, j])) < 1e-6
    td.close()
    tf.close()


@pytest.mark.parametrize("nd,tol", [(6, 1e-6), (3, 2e-4)])
@pytest.mark.parametrize("k", [16, 37, 64, 70])
def test_mixed_tensor_core_blocks(nd, tol, k):
    cell, pos, _ = clustered_system(6000, 48, TRICLINIC, n_clusters=4, sigma=0.03)
    Q = _charges(len(pos), k, 6)
    t = pd.PeriodicDMKTree(cell, pos, nd, 40, 4)
    Pm = _multi_device(t, Q, mixed=True)
    Pd = _multi_device(t, Q, mixed=False)
    errs = [rel_l2(Pm[:, c], Pd[:, c]) for c in range(k)]
    assert max(errs) < tol, (int(np.argmax(errs)), max(errs))
    t.close()


def test_mixed_accuracy_many_sources_per_box():
    # npl 300 at N = 2e5: ~2000 sources per proxy centre and ~250 targets per
    # leaf, the sizes at which long tensor-core accumulations lose accuracy
    cell, pos, _ = uniform_system(200000, 49)
    k = 64
    Q = _charges(len(pos), k, 7)
    tf = pd.PeriodicDMKTree(cell, pos, 6, 300, 4, precision="float")
    td = pd.PeriodicDMKTree(cell, pos, 6, 300, 4)
    Pm = _multi_device(tf, Q, mixed=True)
    for c in (0, 31, 63):
        ref = td.evaluate(Q[:, c])
        assert rel_l2(Pm[:, c], ref) < 1e-6, (c, rel_l2(Pm[:, c], ref))
    tf.close()
    td.close()


def test_float32_charges_equal_double_charges():
    # charges stored in float32 (the 64-RHS workload keeps them in float32 and
    # float64): widened on the device, so on float-representable charges the
    # result equals the double-charge call
    import torch

    cell, pos, _ = uniform_system(4000, 50)
    Q = _charges(len(pos), 16, 8).astype(np.float32)
    t = pd.PeriodicDMKTree(cell, pos, 6, 40, 4, precision="float")
    ref = _multi_device(t, Q.astype(np.float64), mixed=True)
    dev = torch.device("cuda", torch.cuda.current_device())
    q_d = torch.from_numpy(np.ascontiguousarray(Q.T)).to(dev)
    p_d = torch.empty((16, len(pos)), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    t.evaluate_multi_device_f32(16, q_d.data_ptr(), p_d.data_ptr())
    P = p_d.cpu().numpy().T
    H = t.evaluate_multi_f32(Q)
    assert H.dtype == np.float32
    for c in range(16):
        assert rel_l2(P[:, c], ref[:, c]) < 1e-12
        assert rel_l2(H[:, c], ref[:, c]) < 1e-7
    t.close()


@pytest.mark.parametrize("nd,tol", [(6, 5e-6), (3, 2e-4)])
def test_tensor_core_transforms(nd, tol, monkeypatch):
    # PDMK_TC_MASK bit 3 (read when the tree is built) runs the translation and
    # plane-wave transform steps as tcgen05 contractions (3xTF32), against the
    # FP64 path.  3xTF32 keeps about 22 bits of each operand (an 11-bit hi part
    # and an 11-bit rounding of the remainder) against FP32's 24, so its error is
    # a few times that of the CUDA-core FP32 transforms (which keep the 1e-6 bar,
    # test_mixed_multi_accuracy); the 6-digit bar here is 5e-6.  The path is off
    # by default: it is also slower.
    cell, pos, _ = clustered_system(6000, 48, TRICLINIC, n_clusters=4, sigma=0.03)
    Q = _charges(len(pos), 64, 6)
    td = pd.PeriodicDMKTree(cell, pos, nd, 40, 4)
    Pd = _multi_device(td, Q, mixed=False)
    Pc = _multi_device(td, Q, mixed=True)
    td.close()
    monkeypatch.setenv("PDMK_TC_MASK", "15")
    t = pd.PeriodicDMKTree(cell, pos, nd, 40, 4)
    Pm = _multi_device(t, Q, mixed=True)
    t.close()
    errs = [rel_l2(Pm[:, c], Pd[:, c]) for c in range(64)]
    errs_cc = [rel_l2(Pc[:, c], Pd[:, c]) for c in range(64)]
    print("PARITY " + json.dumps({"case": "tcgen05 transforms %d digits" % nd, "max_rel_l2_tc": max(errs),
                                  "max_rel_l2_cuda_core": max(errs_cc)}))
    assert max(errs) < tol, (int(np.argmax(errs)), max(errs))


@pytest.mark.parametrize("precision", ["float", "double"])
def test_overlapped_upload_equals_one_upload(precision, monkeypatch):
    # Host-buffer calls with k a multiple of 8 (and >= 16) upload the charges in
    # 8-column chunks and run each chunk's far field on a second stream while
    # the next chunk is copied; the tree passes start after the last chunk.
    # Against the same call with one upload and the stages in sequence
    # (PDMK_E2E_OVERLAP=0): the far field's FFTs run in batches of 8 instead of
    # k, everything else is the same arithmetic.
    cell, pos, _ = clustered_system(30000, 61, TRICLINIC, n_clusters=4, sigma=0.02)
    Q = _charges(len(pos), 24, 62)
    res = {}
    for ov in ("0", "1"):
        monkeypatch.setenv("PDMK_E2E_OVERLAP", ov)
        t = pd.PeriodicDMKTree(cell, pos, 6, 60, 4, precision=precision)
        a = t.evaluate_multi(Q)
        b = t.evaluate_multi(Q)  # a second call reuses the chunk plans and streams
        f = t.evaluate_multi_f32(Q.astype(np.float32)) if precision == "float" else None
        res[ov] = (a, b, f)
        t.close()
    a0, _, f0 = res["0"]
    a1, b1, f1 = res["1"]
    for c in range(Q.shape[1]):
        assert rel_l2(a1[:, c], a0[:, c]) < 1e-12
        assert rel_l2(b1[:, c], a1[:, c]) < 1e-12
        if f0 is not None:
            assert rel_l2(f1[:, c], f0[:, c]) < 1e-6
    # a width that is not a multiple of 8 takes the one-upload path
    monkeypatch.setenv("PDMK_E2E_OVERLAP", "1")
    t = pd.PeriodicDMKTree(cell, pos, 6, 60, 4, precision=precision)
    c = t.evaluate_multi(Q[:, :19])
    t.close()
    tol = 1e-12 if precision == "double" else 2e-7  # FP32 blocks of another width
    for j in range(19):
        assert rel_l2(c[:, j], a0[:, j]) < tol
