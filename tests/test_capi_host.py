"""CPU tests of the C-ABI library: it loads, exports every declared symbol, and
the host-side entry points and error conventions behave (no GPU needed).
Error conventions follow cpp/src/pdmk_capi.cpp:48-77: create returns NULL on
error, evaluate returns -1 on a null handle."""
import ctypes
import os
import re

import numpy as np
import pytest

import periodicdmk_b200 as pd
from conftest import TRICLINIC, uniform_system

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "pdmk", "pdmk_capi.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(pdmk_[a-z0-9_]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    lib = pd.library()
    declared = _declared_symbols()
    assert len(declared) >= 18
    for name in declared:
        assert hasattr(lib, name), name
    assert sorted(pd.EXPORTED_SYMBOLS) == declared


def test_reference_symbols_present():
    # the entry points the Julia bindings ccall (julia/PeriodicDMK/src/PeriodicDMK.jl)
    for name in ["pdmk_create_double", "pdmk_create_float", "pdmk_evaluate_double", "pdmk_evaluate_float",
                 "pdmk_destroy_double", "pdmk_destroy_float", "pdmk_ewald_nufft", "pdmk_optimize_cubic_cover"]:
        assert name in _declared_symbols()


def test_create_rejects_bad_input_without_device():
    lib = pd.library()
    cell = np.ascontiguousarray(np.eye(3).T).reshape(-1)
    pos = np.zeros(3)
    D = ctypes.POINTER(ctypes.c_double)
    # N = 0
    assert not lib.pdmk_create_double(cell.ctypes.data_as(D), 0, pos.ctypes.data_as(D), 6, 300, 4)
    assert "N must be positive" in pd._last_error()
    # unsupported digit count
    p = np.random.default_rng(0).uniform(0, 1, (10, 3))
    assert not lib.pdmk_create_double(cell.ctypes.data_as(D), 10, p.ctypes.data_as(D), 13, 300, 4)
    assert "n_digits" in pd._last_error()
    # nz <= 0 (automatic rc choice not supported)
    assert not lib.pdmk_create_float(cell.ctypes.data_as(D), 10, p.ctypes.data_as(D), 6, 300, 0)
    assert "nz" in pd._last_error()


def test_null_handle_returns_minus_one():
    lib = pd.library()
    q = np.zeros(4)
    out = np.zeros(4)
    D = ctypes.POINTER(ctypes.c_double)
    assert lib.pdmk_evaluate_double(None, 4, None, q.ctypes.data_as(D), out.ctypes.data_as(D)) == -1
    assert lib.pdmk_evaluate_device_double(None, None, None) == -1
    lib.pdmk_destroy_double(None)  # no-op


def test_python_wrapper_validates_shapes():
    with pytest.raises(ValueError):
        pd.PeriodicDMKTree(np.eye(3), np.zeros((5, 2)))
    with pytest.raises(ValueError):
        pd.PeriodicDMKTree(np.eye(2), np.zeros((5, 3)))


def test_no_cpu_fallback():
    # Without a GPU the CUDA path must fail loudly rather than compute on the host.
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("GPU present")
    cell, pos, q = uniform_system(200, 1)
    with pytest.raises(RuntimeError, match="CUDA"):
        pd.PeriodicDMKTree(cell, pos, 6, 20, 4)


def test_cubic_cover():
    r = pd.optimize_cubic_cover(np.eye(3) * 2.0, nz=4)
    assert (r["m"], r["n"], r["p"]) == (4, 4, 4)
    assert abs(r["s"] - 0.5) < 1e-15
    assert abs(r["cost"] - (6 ** 3 * 0.125) / 8.0) < 1e-12
    np.testing.assert_allclose(np.cross(r["e1"], r["e2"]), r["e3"], atol=1e-15)
    r = pd.optimize_cubic_cover(TRICLINIC, nz=4)
    assert r["p"] == 4 and r["m"] >= 4 and r["n"] >= 4
    with pytest.raises(RuntimeError):
        pd.optimize_cubic_cover(np.eye(3), nz=0)


def test_batch_create_rejects_bad_input_without_compute():
    import ctypes
    lib = pd.library()
    cells = np.tile(np.eye(3).reshape(-1), 2)
    Ns = np.array([10, 0], dtype=np.int32)
    pos = np.zeros(30)
    h = lib.pdmk_batch_create(2, cells.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                              Ns.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                              pos.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 6, 300, 4)
    assert not h
    assert "at least one point" in pd._last_error()
    h = lib.pdmk_batch_create(0, None, None, None, 6, 300, 4)
    assert not h
    assert lib.pdmk_batch_evaluate(None, None, None) == -1


def test_plan_digest_host_construction():
    # the host form of the tree construction (no GPU needed): deterministic,
    # and sensitive to the build parameters
    cell, pos, _ = uniform_system(3000, 7, TRICLINIC)
    d1, _ = pd.plan_digest(cell, pos, 6, 50, 4)
    d2, _ = pd.plan_digest(cell, pos, 6, 50, 4)
    d3, _ = pd.plan_digest(cell, pos, 6, 10, 4)
    assert d1 == d2 and d1 != d3 and len(d1) == 64
