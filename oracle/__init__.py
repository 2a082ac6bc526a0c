"""CPU oracle for the periodic DMK evaluate path (test infrastructure only).

The product never imports this package.  Tests, the smoke check and the
CPU-baseline leg of bench.py load it as the checker.  It wraps
``oracle/_build/liboracle.so`` (built by ``make -C oracle``), a CPU restatement
of the reference evaluate path plus a direct Ewald sum.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build():
    subprocess.run(["make", "-C", _HERE], check=True, stdout=subprocess.DEVNULL)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        d = ctypes.POINTER(ctypes.c_double)
        _lib.oracle_evaluate.argtypes = [d, ctypes.c_int, d, d, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, d, d]
        _lib.oracle_evaluate.restype = ctypes.c_int
        _lib.oracle_evaluate2.argtypes = [d, ctypes.c_int, d, d, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_int, d, d]
        _lib.oracle_evaluate2.restype = ctypes.c_int
        _lib.oracle_plan_stats.argtypes = [d, ctypes.c_int, d, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]
        _lib.oracle_plan_stats.restype = ctypes.c_int
        _lib.oracle_ewald_direct.argtypes = [d, ctypes.c_int, d, d, ctypes.c_double, d, d]
        _lib.oracle_ewald_direct.restype = ctypes.c_int
        ip = ctypes.POINTER(ctypes.c_int)
        _lib.oracle_ewald_targets.argtypes = [d, ctypes.c_int, d, d, ctypes.c_int, ip, ctypes.c_double,
                                              ctypes.c_double, d]
        _lib.oracle_ewald_targets.restype = ctypes.c_int
        _lib.oracle_ewald_targets_grad.argtypes = [d, ctypes.c_int, d, d, ctypes.c_int, ip, ctypes.c_double,
                                                   ctypes.c_double, d, d]
        _lib.oracle_ewald_targets_grad.restype = ctypes.c_int
        _lib.oracle_ewald_targets_qp.argtypes = [d, ctypes.c_int, d, d, ctypes.c_int, ip, ctypes.c_double,
                                                 ctypes.c_double, d, d, d]
        _lib.oracle_ewald_targets_qp.restype = ctypes.c_int
        _lib.oracle_evaluate_multi.argtypes = [d, ctypes.c_int, d, ctypes.c_int, d, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_int, d]
        _lib.oracle_evaluate_multi.restype = ctypes.c_int
        _lib.oracle_tree_compare.argtypes = [d, ctypes.c_int, d, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_longlong)]
        _lib.oracle_tree_compare.restype = ctypes.c_int
        _lib.oracle_plan_new.argtypes = [d, ctypes.c_int, d, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        _lib.oracle_plan_new.restype = ctypes.c_void_p
        _lib.oracle_plan_eval.argtypes = [ctypes.c_void_p, d, ctypes.c_int, ctypes.c_int, d]
        _lib.oracle_plan_eval.restype = ctypes.c_int
        _lib.oracle_plan_free.argtypes = [ctypes.c_void_p]
        _lib.oracle_plan_free.restype = None
        _lib.oracle_pswf.argtypes = [ctypes.c_double, ctypes.c_int, d, d, d]
        _lib.oracle_legendre.argtypes = [ctypes.c_int, d, d]
        ip = ctypes.POINTER(ctypes.c_int)
        _lib.oracle_plan_images.argtypes = [d, ctypes.c_int, d, ctypes.c_int, d, d, ip, d, d, ip, ctypes.c_long]
        _lib.oracle_plan_images.restype = ctypes.c_long
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _cell(cell):
    """cell: 3x3 array whose COLUMNS are lattice vectors -> cell[j*3+i] layout."""
    c = np.asarray(cell, dtype=np.float64)
    return np.ascontiguousarray(c.T).reshape(-1)


def evaluate(cell, pos, q, n_digits=6, n_per_leaf=300, nz=4, with_far=True, components=False, fast_far=False):
    """Oracle potentials.  pos: (N,3) Cartesian, q: (N,).

    The far field is the exact reciprocal-lattice sum unless fast_far=True (CPU
    NUFFT, used for CPU timing only).  Returns pot (N,) or, with
    components=True, (pot, dict(near, mid, self, far)).
    """
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    n = len(q)
    pot = np.zeros(n)
    comp = np.zeros(4 * n)
    c = _cell(cell)
    rc = lib().oracle_evaluate2(_dp(c), n, _dp(pos), _dp(q), n_digits, n_per_leaf, nz,
                                1 if with_far else 0, 1 if fast_far else 0, _dp(pot), _dp(comp))
    if rc != 0:
        raise RuntimeError("oracle_evaluate failed")
    if components:
        comp = comp.reshape(4, n)
        return pot, dict(near=comp[0], mid=comp[1], self=comp[2], far=comp[3])
    return pot


class Plan:
    """Build-once / evaluate-many oracle: the plan (tree, lists, tables) is built
    at construction, evaluate(q) runs only the evaluate stages."""

    def __init__(self, cell, pos, n_digits=6, n_per_leaf=300, nz=4):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        self.n = len(pos)
        c = _cell(cell)
        self._h = lib().oracle_plan_new(_dp(c), self.n, _dp(pos), n_digits, n_per_leaf, nz)
        if not self._h:
            raise RuntimeError("oracle_plan_new failed")

    def evaluate(self, q, with_far=True, fast_far=False):
        q = np.ascontiguousarray(q, dtype=np.float64)
        pot = np.zeros(self.n)
        if lib().oracle_plan_eval(self._h, _dp(q), 1 if with_far else 0, 1 if fast_far else 0, _dp(pot)) != 0:
            raise RuntimeError("oracle_plan_eval failed")
        return pot

    def close(self):
        if self._h:
            lib().oracle_plan_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def plan_stats(cell, pos, n_digits=6, n_per_leaf=300, nz=4):
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    out = (ctypes.c_longlong * 10)()
    c = _cell(cell)
    if lib().oracle_plan_stats(_dp(c), len(pos), _dp(pos), n_digits, n_per_leaf, nz, out) != 0:
        raise RuntimeError("oracle_plan_stats failed")
    keys = ["n_all", "nboxes", "nlevels", "n_target_leaves", "n_pw_boxes", "n_c2proxy_work",
            "n_list1", "ms", "mt", "mu"]
    return dict(zip(keys, list(out)))


def ewald_direct(cell, pos, q, s=5.0):
    """Direct Ewald sum: returns (potentials, energy)."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    pot = np.zeros(len(q))
    e = np.zeros(1)
    c = _cell(cell)
    if lib().oracle_ewald_direct(_dp(c), len(q), _dp(pos), _dp(q), s, _dp(pot), _dp(e)) != 0:
        raise RuntimeError("oracle_ewald_direct failed")
    return pot, float(e[0])


def tree_compare(cell, pos, n_digits=6, n_per_leaf=300, nz=4):
    """Build the tree with the oracle's independent builder (oracle_tree.cpp)
    and compare it with the product's host plan; returns counts and mismatches."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    out = (ctypes.c_longlong * 16)()
    c = _cell(cell)
    if lib().oracle_tree_compare(_dp(c), len(pos), _dp(pos), n_digits, n_per_leaf, nz, out) != 0:
        raise RuntimeError("oracle_tree_compare failed")
    keys = ["boxes", "levels", "leaves_with_sources", "box_mismatch", "leaf_source_mismatch",
            "leaf_target_mismatch", "pwexp_mismatch", "list1_mismatch", "list1_entries", "c2proxy_mismatch",
            "direct_work_mismatch", "image_count_mismatch", "geometry_mismatch", "boxes_l0", "boxes_l1", "boxes_l2"]
    return dict(zip(keys, list(out)))


def ewald_targets(cell, pos, q, targets, s=6.0, alpha=0.0):
    """Ewald potentials at the given target indices (all sources, all images).

    s sets the accuracy (real-space terms below erfc(s), reciprocal terms
    below exp(-s^2)); alpha <= 0 balances the real- and reciprocal-space work.
    Cost ~ len(targets) * (sources within s/alpha) + N * (modes within 2 s alpha).
    """
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    t = np.ascontiguousarray(targets, dtype=np.int32)
    out = np.zeros(len(t))
    c = _cell(cell)
    ip = ctypes.POINTER(ctypes.c_int)
    if lib().oracle_ewald_targets(_dp(c), len(q), _dp(pos), _dp(q), len(t), t.ctypes.data_as(ip), s, alpha,
                                  _dp(out)) != 0:
        raise RuntimeError("oracle_ewald_targets failed")
    return out


def ewald_targets_grad(cell, pos, q, targets, s=6.0, alpha=0.0):
    """(potentials, gradients (m, 3)) at the target indices: Ewald, all sources and
    images; gradient = d phi / d x (Cartesian)."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    t = np.ascontiguousarray(targets, dtype=np.int32)
    out = np.zeros(len(t))
    g = np.zeros(3 * len(t))
    c = _cell(cell)
    ip = ctypes.POINTER(ctypes.c_int)
    if lib().oracle_ewald_targets_grad(_dp(c), len(q), _dp(pos), _dp(q), len(t), t.ctypes.data_as(ip), s, alpha,
                                       _dp(out), _dp(g)) != 0:
        raise RuntimeError("oracle_ewald_targets_grad failed")
    return out, g.reshape(-1, 3)


def ewald_targets_qp(cell, pos, q, targets, bloch, s=6.0, alpha=0.0):
    """Quasi-periodic Ewald potentials (complex) at the target indices: images at
    x_j + R carry e^{i bloch.R} (bloch Cartesian, the caller's frame)."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    t = np.ascontiguousarray(targets, dtype=np.int32)
    b = np.ascontiguousarray(bloch, dtype=np.float64)
    re, im = np.zeros(len(t)), np.zeros(len(t))
    c = _cell(cell)
    ip = ctypes.POINTER(ctypes.c_int)
    if lib().oracle_ewald_targets_qp(_dp(c), len(q), _dp(pos), _dp(q), len(t), t.ctypes.data_as(ip), s, alpha,
                                     _dp(b), _dp(re), _dp(im)) != 0:
        raise RuntimeError("oracle_ewald_targets_qp failed")
    return re + 1j * im


def evaluate_multi(cell, pos, Q, n_digits=6, n_per_leaf=300, nz=4):
    """Oracle potentials of k charge vectors Q (N, k) on one plan (exact far field)."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    Qc = np.ascontiguousarray(np.asarray(Q, dtype=np.float64).T)  # column-major N x k
    n, k = Qc.shape[1], Qc.shape[0]
    out = np.zeros_like(Qc)
    c = _cell(cell)
    if lib().oracle_evaluate_multi(_dp(c), n, _dp(pos), k, _dp(Qc), n_digits, n_per_leaf, nz, _dp(out)) != 0:
        raise RuntimeError("oracle_evaluate_multi failed")
    return out.T


def pswf(beta, x):
    """Host PSWF psi_0^beta(x) and moments (c0, c1, c2/c0, c4) of the product's plan builder."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    psi = np.zeros_like(x)
    m = np.zeros(4)
    lib().oracle_pswf(beta, len(x), _dp(x), _dp(psi), _dp(m))
    return psi, m


def legendre(n):
    x, w = np.zeros(n), np.zeros(n)
    lib().oracle_legendre(n, _dp(x), _dp(w))
    return x, w


def plan_images(cell, pos, nz=4):
    """(umat, qmat, mgrid, xgrid0, rc, img_src_idx) of the product's host plan."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    c = _cell(cell)
    umat, qmat, xg, rc = np.zeros(9), np.zeros(9), np.zeros(3), np.zeros(1)
    mg = np.zeros(3, dtype=np.int32)
    cap = 60 * len(pos)
    idx = np.zeros(cap, dtype=np.int32)
    ip = ctypes.POINTER(ctypes.c_int)
    n = lib().oracle_plan_images(_dp(c), len(pos), _dp(pos), nz, _dp(umat), _dp(qmat), mg.ctypes.data_as(ip),
                                 _dp(xg), _dp(rc), idx.ctypes.data_as(ip), cap)
    if n < 0:
        raise RuntimeError("oracle_plan_images failed")
    return umat, qmat, mg, xg, float(rc[0]), idx[:n]
