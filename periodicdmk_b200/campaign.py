"""Campaign reference files ('PDMC' format): oracle potentials at M sampled
points of an N-point periodic system, stored with the system (cell, positions,
charges) and guarded by a SHA-256 of the body.  Byte-compatible with the
reference's cpp/include/pdmk/campaign_ref_io.hpp (written and read through
libpdmk_b200.so: pdmk_campaign_write / pdmk_campaign_read).
"""
import ctypes

import numpy as np

from . import _last_error, _ptr, library

__all__ = ["sha256", "write_ref", "read_ref", "DEFAULT_M"]

DEFAULT_M = 1000
_U32 = ctypes.POINTER(ctypes.c_uint32)


def sha256(data):
    """SHA-256 digest (32 bytes) of a bytes-like object, computed by the library."""
    buf = bytes(data)
    out = ctypes.create_string_buffer(32)
    src = ctypes.c_char_p(buf) if buf else None
    if library().pdmk_sha256(src, len(buf), out) != 0:
        raise RuntimeError("pdmk_sha256 failed: " + _last_error())
    return out.raw


def write_ref(path, cell, positions, charges, ref_idx, ref_u, config_id=0, digits=6, prec=1, seed=0):
    """Write a reference file.  cell: 3x3 with the lattice vectors as columns;
    positions (N, 3); charges (N,); ref_idx (M,) point indices; ref_u (M,)
    reference potentials at those points."""
    c = np.ascontiguousarray(np.asarray(cell, dtype=np.float64).reshape(3, 3).T.ravel())  # column-major
    pos = np.ascontiguousarray(positions, dtype=np.float64)
    if pos.ndim != 2 or pos.shape[1] != 3:
        raise ValueError("positions must be (N, 3)")
    q = np.ascontiguousarray(charges, dtype=np.float64)
    idx = np.ascontiguousarray(ref_idx, dtype=np.uint32)
    u = np.ascontiguousarray(ref_u, dtype=np.float64)
    n = pos.shape[0]
    if q.shape != (n,) or idx.shape != u.shape or idx.ndim != 1:
        raise ValueError("charges must be (N,), ref_idx and ref_u (M,)")
    if idx.size and int(idx.max()) >= n:
        raise ValueError("ref_idx out of range")
    rc = library().pdmk_campaign_write(path.encode(), int(config_id), int(digits), int(prec), int(seed), _ptr(c), n,
                                       _ptr(pos), _ptr(q), idx.size, idx.ctypes.data_as(_U32), _ptr(u))
    if rc != 0:
        raise RuntimeError("pdmk_campaign_write failed: " + _last_error())


def read_ref(path):
    """Read and check a reference file: dict with config_id, N, M, digits, prec,
    seed, cell (3x3, lattice vectors as columns), positions (N, 3), charges,
    ref_idx, ref_u.  Raises on a malformed file or a digest mismatch."""
    lib = library()
    hdr = np.zeros(5, dtype=np.uint32)
    seed = ctypes.c_uint64(0)
    if lib.pdmk_campaign_read_header(path.encode(), hdr.ctypes.data_as(_U32), ctypes.byref(seed)) != 0:
        raise RuntimeError("pdmk_campaign_read_header failed: " + _last_error())
    n, m = int(hdr[1]), int(hdr[2])
    cell = np.zeros(9)
    pos = np.zeros((max(n, 1), 3))
    q = np.zeros(max(n, 1))
    idx = np.zeros(max(m, 1), dtype=np.uint32)
    u = np.zeros(max(m, 1))
    if lib.pdmk_campaign_read(path.encode(), _ptr(cell), _ptr(pos), _ptr(q), idx.ctypes.data_as(_U32), _ptr(u)) != 0:
        raise RuntimeError("pdmk_campaign_read failed: " + _last_error())
    return dict(config_id=int(hdr[0]), N=n, M=m, digits=int(hdr[3]), prec=int(hdr[4]), seed=int(seed.value),
                cell=cell.reshape(3, 3).T.copy(), positions=pos[:n], charges=q[:n], ref_idx=idx[:m], ref_u=u[:m])
