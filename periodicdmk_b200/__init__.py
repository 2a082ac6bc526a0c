"""B200-native periodic DMK (3D Laplace / Coulomb) evaluate path.

Python mirror of the reference's build-once / evaluate-many interface
(``PeriodicDMKTreeT`` in cpp/include/pdmk/periodic_dmk.hpp:17-60 and the Julia
``PDMKSolver`` in julia/PeriodicDMK/src/PeriodicDMK.jl:90-211), bound to the
C ABI of ``lib/libpdmk_b200.so`` (include/pdmk/pdmk_capi.h).  Every evaluate
runs on the GPU; there is no CPU fallback: if the library cannot be loaded,
or CUDA is unavailable, the calls raise.
"""
import ctypes
import os

import numpy as np

__all__ = ["PeriodicDMKTree", "PeriodicDMKBatch", "library", "library_path", "ewald", "optimize_cubic_cover",
           "EXPORTED_SYMBOLS"]

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "lib", "libpdmk_b200.so")
_lib = None

# Every entry point declared in include/pdmk/pdmk_capi.h.
EXPORTED_SYMBOLS = [
    "pdmk_ewald_nufft", "pdmk_optimize_cubic_cover",
    "pdmk_create_double", "pdmk_create_float",
    "pdmk_evaluate_double", "pdmk_evaluate_float",
    "pdmk_destroy_double", "pdmk_destroy_float",
    "pdmk_evaluate_timed_double", "pdmk_evaluate_timed_float",
    "pdmk_evaluate_multi_double", "pdmk_evaluate_multi_float",
    "pdmk_evaluate_device_double", "pdmk_evaluate_device_float",
    "pdmk_evaluate_multi_device_double", "pdmk_evaluate_multi_device_float",
    "pdmk_evaluate_multi_float_qf32", "pdmk_evaluate_multi_device_float_qf32",
    "pdmk_evaluate_grad_double", "pdmk_evaluate_grad_device_double",
    "pdmk_evaluate_parts_double", "pdmk_info_double", "pdmk_info_float",
    "pdmk_stage_times_double", "pdmk_stage_times_float", "pdmk_fma_peak", "pdmk_tc_peak",
    "pdmk_evaluate_device_noalloc_double",
    "pdmk_create_qp_double", "pdmk_create_qp_float", "pdmk_evaluate_complex_double",
    "pdmk_evaluate_complex_float", "pdmk_evaluate_complex_device_double",
    "pdmk_batch_create", "pdmk_batch_create_double", "pdmk_batch_evaluate", "pdmk_batch_evaluate_float",
    "pdmk_batch_info", "pdmk_batch_destroy",
    "pdmk_sha256", "pdmk_campaign_write", "pdmk_campaign_read_header", "pdmk_campaign_read", "pdmk_plan_digest",
    "pdmk_last_error",
]

_D = ctypes.POINTER(ctypes.c_double)
_F = ctypes.POINTER(ctypes.c_float)
_I64 = ctypes.POINTER(ctypes.c_int64)
_I = ctypes.POINTER(ctypes.c_int)


def library_path():
    return _LIB_PATH


def library():
    """Load libpdmk_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise ImportError("libpdmk_b200.so not built: run `python -m periodicdmk_b200.build` (%s)" % _LIB_PATH)
    lib = ctypes.CDLL(_LIB_PATH)
    v = ctypes.c_void_p
    lib.pdmk_create_double.argtypes = [_D, ctypes.c_int, _D, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.pdmk_create_double.restype = v
    lib.pdmk_create_float.argtypes = lib.pdmk_create_double.argtypes
    lib.pdmk_create_float.restype = v
    lib.pdmk_create_qp_double.argtypes = [_D, ctypes.c_int, _D, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D]
    lib.pdmk_create_qp_double.restype = v
    lib.pdmk_create_qp_float.argtypes = lib.pdmk_create_qp_double.argtypes
    lib.pdmk_create_qp_float.restype = v
    lib.pdmk_evaluate_complex_double.argtypes = [v, ctypes.c_int, _D, _D, _D]
    lib.pdmk_evaluate_complex_double.restype = ctypes.c_int
    lib.pdmk_evaluate_complex_float.argtypes = [v, ctypes.c_int, _D, _D, _F]
    lib.pdmk_evaluate_complex_float.restype = ctypes.c_int
    lib.pdmk_evaluate_complex_device_double.argtypes = [v, ctypes.c_void_p, ctypes.c_void_p]
    lib.pdmk_evaluate_complex_device_double.restype = ctypes.c_int
    lib.pdmk_evaluate_double.argtypes = [v, ctypes.c_int, _D, _D, _D]
    lib.pdmk_evaluate_float.argtypes = [v, ctypes.c_int, _D, _D, _F]
    lib.pdmk_evaluate_timed_double.argtypes = [v, ctypes.c_int, _D, _D, _D, _D]
    lib.pdmk_evaluate_timed_float.argtypes = [v, ctypes.c_int, _D, _D, _F, _D]
    lib.pdmk_evaluate_multi_double.argtypes = [v, ctypes.c_int, ctypes.c_int, _D, _D]
    lib.pdmk_evaluate_multi_float.argtypes = [v, ctypes.c_int, ctypes.c_int, _D, _F]
    lib.pdmk_evaluate_device_double.argtypes = [v, ctypes.c_void_p, ctypes.c_void_p]
    lib.pdmk_evaluate_device_float.argtypes = [v, ctypes.c_void_p, ctypes.c_void_p]
    lib.pdmk_evaluate_parts_double.argtypes = [v, _D, _D, _D]
    lib.pdmk_evaluate_multi_device_double.argtypes = [v, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    lib.pdmk_evaluate_multi_device_double.restype = ctypes.c_int
    lib.pdmk_evaluate_multi_device_float.argtypes = [v, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    lib.pdmk_evaluate_multi_device_float.restype = ctypes.c_int
    lib.pdmk_evaluate_multi_float_qf32.argtypes = [v, ctypes.c_int, ctypes.c_int, _F, _F]
    lib.pdmk_evaluate_grad_double.argtypes = [v, ctypes.c_int, _D, _D, _D, _D]
    lib.pdmk_evaluate_grad_double.restype = ctypes.c_int
    lib.pdmk_evaluate_grad_device_double.argtypes = [v, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.pdmk_evaluate_grad_device_double.restype = ctypes.c_int
    lib.pdmk_evaluate_multi_device_float_qf32.argtypes = [v, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    lib.pdmk_info_double.argtypes = [v, _I64]
    lib.pdmk_info_float.argtypes = [v, _I64]
    for f in ("pdmk_evaluate_double", "pdmk_evaluate_float", "pdmk_evaluate_timed_double",
              "pdmk_evaluate_timed_float", "pdmk_evaluate_multi_double", "pdmk_evaluate_multi_float",
              "pdmk_evaluate_device_double", "pdmk_evaluate_device_float",
              "pdmk_evaluate_multi_device_double", "pdmk_evaluate_multi_device_float",
              "pdmk_evaluate_multi_float_qf32", "pdmk_evaluate_multi_device_float_qf32",
              "pdmk_evaluate_parts_double", "pdmk_info_double", "pdmk_info_float"):
        getattr(lib, f).restype = ctypes.c_int
    lib.pdmk_destroy_double.argtypes = [v]
    lib.pdmk_destroy_double.restype = None
    lib.pdmk_destroy_float.argtypes = [v]
    lib.pdmk_destroy_float.restype = None
    lib.pdmk_ewald_nufft.argtypes = [_D, ctypes.c_int, _D, _D, ctypes.c_double, _D, _D]
    lib.pdmk_ewald_nufft.restype = ctypes.c_int
    lib.pdmk_optimize_cubic_cover.argtypes = [_D, ctypes.c_int, _I, _I, _I, _D, _D, _D, _D, _D]
    lib.pdmk_optimize_cubic_cover.restype = ctypes.c_int
    lib.pdmk_stage_times_double.argtypes = [v, _D]
    lib.pdmk_stage_times_double.restype = ctypes.c_int
    lib.pdmk_stage_times_float.argtypes = [v, _D]
    lib.pdmk_stage_times_float.restype = ctypes.c_int
    lib.pdmk_evaluate_device_noalloc_double.argtypes = [v, ctypes.c_void_p, ctypes.c_void_p]
    lib.pdmk_evaluate_device_noalloc_double.restype = ctypes.c_int
    lib.pdmk_fma_peak.argtypes = [ctypes.c_int, _D]
    lib.pdmk_fma_peak.restype = ctypes.c_int
    lib.pdmk_tc_peak.argtypes = [ctypes.c_int, _D]
    lib.pdmk_tc_peak.restype = ctypes.c_int
    lib.pdmk_batch_create.argtypes = [ctypes.c_int, _D, _I, _D, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.pdmk_batch_create.restype = v
    lib.pdmk_batch_create_double.argtypes = lib.pdmk_batch_create.argtypes
    lib.pdmk_batch_create_double.restype = v
    lib.pdmk_batch_evaluate.argtypes = [v, _D, _D]
    lib.pdmk_batch_evaluate.restype = ctypes.c_int
    lib.pdmk_batch_evaluate_float.argtypes = [v, _D, _F]
    lib.pdmk_batch_evaluate_float.restype = ctypes.c_int
    lib.pdmk_batch_info.argtypes = [v, _I64]
    lib.pdmk_batch_info.restype = ctypes.c_int
    lib.pdmk_batch_destroy.argtypes = [v]
    lib.pdmk_batch_destroy.restype = None
    u32p = ctypes.POINTER(ctypes.c_uint32)
    lib.pdmk_sha256.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
    lib.pdmk_sha256.restype = ctypes.c_int
    lib.pdmk_campaign_write.argtypes = [ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                        ctypes.c_uint64, _D, ctypes.c_uint32, _D, _D, ctypes.c_uint32, u32p, _D]
    lib.pdmk_campaign_write.restype = ctypes.c_int
    lib.pdmk_campaign_read_header.argtypes = [ctypes.c_char_p, u32p, ctypes.POINTER(ctypes.c_uint64)]
    lib.pdmk_campaign_read_header.restype = ctypes.c_int
    lib.pdmk_campaign_read.argtypes = [ctypes.c_char_p, _D, _D, _D, u32p, _D]
    lib.pdmk_campaign_read.restype = ctypes.c_int
    lib.pdmk_plan_digest.argtypes = [_D, ctypes.c_int, _D, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_void_p, _D]
    lib.pdmk_plan_digest.restype = ctypes.c_int
    lib.pdmk_last_error.argtypes = []
    lib.pdmk_last_error.restype = ctypes.c_char_p
    _lib = lib
    return lib


def _last_error():
    return library().pdmk_last_error().decode(errors="replace")


def _ptr(a, t=_D):
    return a.ctypes.data_as(t)


def _cell_colmajor(cell):
    """3x3 with lattice vectors as COLUMNS -> column-major flat (cell[i + 3*j])."""
    c = np.asarray(cell, dtype=np.float64)
    if c.shape != (3, 3):
        raise ValueError("cell must be 3x3 (columns = lattice vectors)")
    return np.ascontiguousarray(c.T).reshape(-1)


class PeriodicDMKTree:
    """Build-once / evaluate-many periodic Coulomb solver on one GPU.

    cell: 3x3, columns are the lattice vectors.  positions: (N, 3) Cartesian.
    precision: "double" (plain FP64 path) or "float" (mixed-precision path,
    float output), as the reference's double / float instantiations.
    bloch: optional Bloch vector (3,), in the lattice-QR frame as the
    reference takes it; the tree is then quasi-periodic and evaluates with
    evaluate_complex only (the real evaluates raise).
    """

    INFO_KEYS = ["n_points", "n_all", "n_boxes", "n_levels", "n_target_leaves", "p", "n_pw",
                 "launches_per_evaluate", "device_bytes", "far_modes", "near_pairs", "pw_boxes",
                 "launches_last_multi", "n_digits_tree", "mixed_available", "translate_boxes"]

    def __init__(self, cell, positions, n_digits=6, n_per_leaf=300, nz=4, precision="double", bloch=None):
        if precision not in ("double", "float"):
            raise ValueError("precision must be 'double' or 'float'")
        pos = np.ascontiguousarray(positions, dtype=np.float64)
        if pos.ndim != 2 or pos.shape[1] != 3:
            raise ValueError("positions must be (N, 3)")
        self._lib = library()
        self.precision = precision
        self.N = pos.shape[0]
        c = _cell_colmajor(cell)
        self.bloch = None
        if bloch is None:
            create = self._lib.pdmk_create_double if precision == "double" else self._lib.pdmk_create_float
            self._h = create(_ptr(c), self.N, _ptr(pos), int(n_digits), int(n_per_leaf), int(nz))
        else:
            b = np.ascontiguousarray(bloch, dtype=np.float64)
            if b.shape != (3,):
                raise ValueError("bloch must have shape (3,)")
            self.bloch = b
            create = self._lib.pdmk_create_qp_double if precision == "double" else self._lib.pdmk_create_qp_float
            self._h = create(_ptr(c), self.N, _ptr(pos), int(n_digits), int(n_per_leaf), int(nz), _ptr(b))
        if not self._h:
            raise RuntimeError("pdmk_create failed: " + _last_error())
        self.n_digits = n_digits

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError("%s failed (code %d): %s" % (what, rc, _last_error()))

    def _charges(self, charges):
        q = np.ascontiguousarray(charges, dtype=np.float64)
        if q.shape != (self.N,):
            raise ValueError("charges must have shape (%d,)" % self.N)
        return q

    @property
    def dtype(self):
        return np.float64 if self.precision == "double" else np.float32

    def evaluate(self, charges):
        q = self._charges(charges)
        out = np.empty(self.N, dtype=self.dtype)
        dummy = np.zeros(3, dtype=np.float64)
        if self.precision == "double":
            rc = self._lib.pdmk_evaluate_double(self._h, self.N, _ptr(dummy), _ptr(q), _ptr(out))
        else:
            rc = self._lib.pdmk_evaluate_float(self._h, self.N, _ptr(dummy), _ptr(q), _ptr(out, _F))
        self._check(rc, "pdmk_evaluate")
        return out

    def evaluate_timed(self, charges):
        """Returns (potentials, {"nufft_ms", "dmk_ms", "direct_ms", "build_ms"})."""
        q = self._charges(charges)
        out = np.empty(self.N, dtype=self.dtype)
        t = np.zeros(4)
        dummy = np.zeros(3, dtype=np.float64)
        if self.precision == "double":
            rc = self._lib.pdmk_evaluate_timed_double(self._h, self.N, _ptr(dummy), _ptr(q), _ptr(out), _ptr(t))
        else:
            rc = self._lib.pdmk_evaluate_timed_float(self._h, self.N, _ptr(dummy), _ptr(q), _ptr(out, _F), _ptr(t))
        self._check(rc, "pdmk_evaluate_timed")
        return out, dict(nufft_ms=t[0], dmk_ms=t[1], direct_ms=t[2], build_ms=t[3])

    def evaluate_multi(self, charges):
        """charges: (N, k) -> potentials (N, k)."""
        q = np.asarray(charges, dtype=np.float64)
        if q.ndim != 2 or q.shape[0] != self.N:
            raise ValueError("charges must be (N, k)")
        k = q.shape[1]
        qc = np.ascontiguousarray(q.T)  # column-major N x k
        out = np.empty((k, self.N), dtype=self.dtype)
        if self.precision == "double":
            rc = self._lib.pdmk_evaluate_multi_double(self._h, self.N, k, _ptr(qc), _ptr(out))
        else:
            rc = self._lib.pdmk_evaluate_multi_float(self._h, self.N, k, _ptr(qc), _ptr(out, _F))
        self._check(rc, "pdmk_evaluate_multi")
        return out.T

    def evaluate_device(self, q_ptr, pot_ptr):
        """Device-resident evaluate on raw device pointers (e.g. torch .data_ptr())."""
        f = self._lib.pdmk_evaluate_device_double if self.precision == "double" else \
            self._lib.pdmk_evaluate_device_float
        self._check(f(self._h, ctypes.c_void_p(q_ptr), ctypes.c_void_p(pot_ptr)), "pdmk_evaluate_device")

    def evaluate_device_noalloc(self, q_ptr, pot_ptr):
        """Device-resident evaluate that allocates no device memory (double trees).

        For callers that must not allocate device memory once running (their
        own allocator owns the pool, or cudaMalloc's device-wide
        synchronisation is unacceptable in their loop).  Uses the library's
        static 32 MiB scratch array; overlapping calls on one GPU race."""
        if self.precision != "double":
            raise RuntimeError("evaluate_device_noalloc is provided for double trees")
        rc = self._lib.pdmk_evaluate_device_noalloc_double(self._h, ctypes.c_void_p(q_ptr), ctypes.c_void_p(pot_ptr))
        self._check(rc, "pdmk_evaluate_device_noalloc_double")

    def evaluate_multi_device(self, k, q_ptr, pot_ptr, mixed=None):
        """k charge vectors on device buffers (N x k column-major doubles in and out).

        mixed: True for the mixed-precision path, False for plain FP64 (double
        trees only; float trees always use the mixed path)."""
        if self.precision == "double":
            rc = self._lib.pdmk_evaluate_multi_device_double(self._h, int(k), ctypes.c_void_p(q_ptr),
                                                             ctypes.c_void_p(pot_ptr), 1 if mixed else 0)
        else:
            rc = self._lib.pdmk_evaluate_multi_device_float(self._h, int(k), ctypes.c_void_p(q_ptr),
                                                            ctypes.c_void_p(pot_ptr))
        self._check(rc, "pdmk_evaluate_multi_device")

    def evaluate_complex(self, charges):
        """Quasi-periodic potentials sum_j q_j sum_R e^{i bloch.R} G(x_i - x_j - R)
        of a tree built with a Bloch vector: complex128 (double trees) or
        complex64 (float trees), computed in FP64."""
        q = self._charges(charges)
        dummy = np.zeros(3, dtype=np.float64)
        if self.precision == "double":
            out = np.empty(2 * self.N)
            rc = self._lib.pdmk_evaluate_complex_double(self._h, self.N, _ptr(dummy), _ptr(q), _ptr(out))
        else:
            out = np.empty(2 * self.N, dtype=np.float32)
            rc = self._lib.pdmk_evaluate_complex_float(self._h, self.N, _ptr(dummy), _ptr(q), _ptr(out, _F))
        self._check(rc, "pdmk_evaluate_complex")
        return out.view(np.complex128 if self.precision == "double" else np.complex64)

    def evaluate_complex_device(self, q_ptr, pot2_ptr):
        """Quasi-periodic evaluate on device buffers (N charges; 2N doubles out,
        (Re, Im) interleaved) of a double tree."""
        if self.precision != "double":
            raise RuntimeError("evaluate_complex_device is provided for double trees")
        rc = self._lib.pdmk_evaluate_complex_device_double(self._h, ctypes.c_void_p(q_ptr), ctypes.c_void_p(pot2_ptr))
        self._check(rc, "pdmk_evaluate_complex_device_double")

    def evaluate_grad(self, charges):
        """(potentials (N,), gradients (N, 3)) of a double tree; gradient = d u / d x
        (the field is -gradient)."""
        if self.precision != "double":
            raise ValueError("gradients are computed by double trees")
        q = self._charges(charges)
        pot = np.empty(self.N)
        grad = np.empty((self.N, 3))
        dummy = np.zeros(3, dtype=np.float64)
        rc = self._lib.pdmk_evaluate_grad_double(self._h, self.N, _ptr(dummy), _ptr(q), _ptr(pot), _ptr(grad))
        self._check(rc, "pdmk_evaluate_grad_double")
        return pot, grad

    def evaluate_multi_f32(self, charges):
        """k charge vectors stored as float32 (N, k) on a float tree: float32 in,
        float32 potentials (N, k) out (pdmk_evaluate_multi_float_qf32)."""
        if self.precision != "float":
            raise ValueError("float32 charges are taken by float trees (mixed-precision path)")
        Q = np.asarray(charges, dtype=np.float32)
        if Q.ndim != 2 or Q.shape[0] != self.N:
            raise ValueError("charges must be (N, k)")
        k = Q.shape[1]
        Qc = np.ascontiguousarray(Q.T)  # column-major N x k
        out = np.empty((k, self.N), dtype=np.float32)
        rc = self._lib.pdmk_evaluate_multi_float_qf32(self._h, self.N, k, _ptr(Qc, _F), _ptr(out, _F))
        self._check(rc, "pdmk_evaluate_multi_float_qf32")
        return out.T

    def evaluate_multi_device_f32(self, k, q_ptr, pot_ptr):
        """float32 charges (N x k column-major, device) -> double potentials (device); float trees."""
        rc = self._lib.pdmk_evaluate_multi_device_float_qf32(self._h, int(k), ctypes.c_void_p(q_ptr),
                                                             ctypes.c_void_p(pot_ptr))
        self._check(rc, "pdmk_evaluate_multi_device_float_qf32")

    def evaluate_parts(self, charges):
        """(tree part, far-field part), both user order; double trees only."""
        if self.precision != "double":
            raise RuntimeError("evaluate_parts is provided for double trees")
        q = self._charges(charges)
        a = np.empty(self.N)
        b = np.empty(self.N)
        self._check(self._lib.pdmk_evaluate_parts_double(self._h, _ptr(q), _ptr(a), _ptr(b)),
                    "pdmk_evaluate_parts")
        return a, b

    def info(self):
        out = np.zeros(16, dtype=np.int64)
        f = self._lib.pdmk_info_double if self.precision == "double" else self._lib.pdmk_info_float
        self._check(f(self._h, _ptr(out, _I64)), "pdmk_info")
        return dict(zip(self.INFO_KEYS, [int(x) for x in out]))

    STAGE_KEYS = ["dmk_ms", "near_ms", "nufft_ms", "finalize_ms", "total_ms", "near_pairs_culled",
                  "near_pairs_nominal", "near_ncoef"]

    def stage_times(self):
        """Stage times of the most recent evaluate (multi-RHS: summed over RHS blocks)."""
        out = np.zeros(8)
        f = self._lib.pdmk_stage_times_double if self.precision == "double" else self._lib.pdmk_stage_times_float
        self._check(f(self._h, _ptr(out)), "pdmk_stage_times")
        return dict(zip(self.STAGE_KEYS, out.tolist()))

    def close(self):
        if getattr(self, "_h", None):
            (self._lib.pdmk_destroy_double if self.precision == "double" else self._lib.pdmk_destroy_float)(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class PeriodicDMKBatch:
    """Many independent periodic systems built and evaluated together.

    cells: sequence of 3x3 (columns = lattice vectors); positions: sequence of
    (N_i, 3) arrays.  precision "auto" follows the reference's
    AutoPeriodicDMKTree (float / mixed precision for n_digits <= 6, double
    above); "double" forces double trees.  evaluate takes a sequence of charge
    vectors and returns a list of potential arrays (float64).
    """

    def __init__(self, cells, positions, n_digits=6, n_per_leaf=300, nz=4, precision="auto"):
        if precision not in ("auto", "double"):
            raise ValueError("precision must be 'auto' or 'double'")
        if len(cells) != len(positions) or len(cells) == 0:
            raise ValueError("need one cell per system and at least one system")
        self._lib = library()
        pos = [np.ascontiguousarray(p, dtype=np.float64) for p in positions]
        for p in pos:
            if p.ndim != 2 or p.shape[1] != 3 or p.shape[0] == 0:
                raise ValueError("positions must be non-empty (N_i, 3) arrays")
        self.Ns = np.array([p.shape[0] for p in pos], dtype=np.int32)
        self.offsets = np.concatenate([[0], np.cumsum(self.Ns, dtype=np.int64)])
        c = np.concatenate([_cell_colmajor(cc) for cc in cells])
        allpos = np.ascontiguousarray(np.concatenate(pos, axis=0))
        create = self._lib.pdmk_batch_create if precision == "auto" else self._lib.pdmk_batch_create_double
        self._h = create(len(pos), _ptr(c), _ptr(self.Ns, _I), _ptr(allpos), int(n_digits), int(n_per_leaf), int(nz))
        if not self._h:
            raise RuntimeError("pdmk_batch_create failed: " + _last_error())

    def info(self):
        out = np.zeros(4, dtype=np.int64)
        if self._lib.pdmk_batch_info(self._h, _ptr(out, _I64)) != 0:
            raise RuntimeError("pdmk_batch_info failed: " + _last_error())
        return {"n_systems": int(out[0]), "n_points": int(out[1]), "device_bytes": int(out[2]),
                "float_trees": bool(out[3])}

    def evaluate(self, charges, out_dtype=np.float64, out=None):
        """charges: a sequence of per-system charge vectors, or one float64 array
        of all systems' charges concatenated (used without a copy).  out: an
        optional preallocated array of all potentials (out_dtype, concatenated)
        that is written in place.  Returns the per-system potentials (views of
        the concatenated output)."""
        total = int(self.offsets[-1])
        if isinstance(charges, np.ndarray) and charges.ndim == 1:
            q = np.ascontiguousarray(charges, dtype=np.float64)
        else:
            q = np.ascontiguousarray(np.concatenate([np.asarray(c, dtype=np.float64) for c in charges]))
        if q.shape != (total,):
            raise ValueError("charges must match the systems' point counts")
        out_dtype = np.dtype(out_dtype)
        if out_dtype not in (np.dtype(np.float32), np.dtype(np.float64)):
            raise ValueError("out_dtype must be float32 or float64")
        if out is None:
            out = np.empty(total, dtype=out_dtype)
        elif (not isinstance(out, np.ndarray) or out.shape != (total,) or out.dtype != out_dtype
              or not out.flags.c_contiguous or not out.flags.writeable):
            raise ValueError("out must be a writeable contiguous (total,) array of out_dtype")
        if out_dtype == np.float32:
            rc = self._lib.pdmk_batch_evaluate_float(self._h, _ptr(q), _ptr(out, _F))
        else:
            rc = self._lib.pdmk_batch_evaluate(self._h, _ptr(q), _ptr(out))
        if rc != 0:
            raise RuntimeError("pdmk_batch_evaluate failed (code %d): %s" % (rc, _last_error()))
        return [out[self.offsets[i]:self.offsets[i + 1]] for i in range(len(self.Ns))]

    def close(self):
        if getattr(self, "_h", None):
            self._lib.pdmk_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ewald(cell, positions, charges, s=4.8):
    """Ewald summation on the GPU through the C ABI (pdmk_ewald_nufft: cell-list
    real-space sum, NUFFT reciprocal sum).  Returns (potentials, energy)."""
    lib = library()
    pos = np.ascontiguousarray(positions, dtype=np.float64)
    q = np.ascontiguousarray(charges, dtype=np.float64)
    pot = np.empty(len(q))
    e = np.zeros(1)
    c = _cell_colmajor(cell)
    rc = lib.pdmk_ewald_nufft(_ptr(c), len(q), _ptr(pos), _ptr(q), float(s), _ptr(pot), _ptr(e))
    if rc != 0:
        raise RuntimeError("pdmk_ewald_nufft failed: " + _last_error())
    return pot, float(e[0])


def plan_digest(cell, positions, n_digits=6, n_per_leaf=300, nz=4, on_device=False):
    """(SHA-256 hex of the tree plan, build milliseconds) with the point steps of
    the tree construction on the host or on the GPU; both give the same digest."""
    pos = np.ascontiguousarray(positions, dtype=np.float64)
    c = _cell_colmajor(cell)
    out = ctypes.create_string_buffer(32)
    ms = np.zeros(1)
    rc = library().pdmk_plan_digest(_ptr(c), len(pos), _ptr(pos), int(n_digits), int(n_per_leaf), int(nz),
                                    1 if on_device else 0, out, _ptr(ms))
    if rc != 0:
        raise RuntimeError("pdmk_plan_digest failed: " + _last_error())
    return out.raw.hex(), float(ms[0])


def optimize_cubic_cover(cell, nz=4):
    lib = library()
    c = _cell_colmajor(cell)
    m, n, p = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    e1, e2, e3 = np.zeros(3), np.zeros(3), np.zeros(3)
    s, cost = np.zeros(1), np.zeros(1)
    rc = lib.pdmk_optimize_cubic_cover(_ptr(c), int(nz), ctypes.byref(m), ctypes.byref(n), ctypes.byref(p),
                                       _ptr(e1), _ptr(e2), _ptr(e3), _ptr(s), _ptr(cost))
    if rc != 0:
        raise RuntimeError("pdmk_optimize_cubic_cover failed (code %d)" % rc)
    return dict(m=m.value, n=n.value, p=p.value, e1=e1, e2=e2, e3=e3, s=float(s[0]), cost=float(cost[0]))


def tc_peak_tflops(kind="tf32"):
    """Measured tensor-core throughput of the current CUDA device (TFLOP/s):
    "tf32" = tcgen05 TF32 MMA, "fp64" = FP64 DMMA (mma.sync m8n8k4)."""
    k = {"tf32": 0, "fp64": 1}[kind]
    out = np.zeros(1)
    if library().pdmk_tc_peak(k, _ptr(out)) != 0:
        raise RuntimeError("pdmk_tc_peak failed: " + _last_error())
    return float(out[0])


def fma_peak_tflops(fp64=True):
    """Measured FMA throughput of the current CUDA device (TFLOP/s)."""
    out = np.zeros(1)
    if library().pdmk_fma_peak(1 if fp64 else 0, _ptr(out)) != 0:
        raise RuntimeError("pdmk_fma_peak failed: " + _last_error())
    return float(out[0])
