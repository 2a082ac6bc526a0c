"""Generate the golden fixtures in tests/golden/ from the reference's own code.

Runs only where the reference source tree is present (PDMK_REFERENCE_DIR names
the reference project's root): it builds
oracle/_ref/libref.so from the reference's standalone sources
(cpp/src/dmk/prolate.cpp, cpp/src/dmk/legeexps.cpp, cpp/include/dmk/pbc.hpp,
cpp/include/pdmk/image_layout.hpp) with `make -C oracle ref` and records:
  pswf.json    psi_0^beta on a grid of x and the moments (c0, c1, c2, c4) for the
               four bandwidths of the 3/6/9/12-digit brackets
  legendre.json  the reference's 100- and 200-point Gauss-Legendre rules
  images.json  lattice QR, grid and image layout (count + index checksum) for
               seeded systems of the path's configurations
The fixtures are committed; tests compare the oracle and the product's host
code against them without needing the reference.

    PDMK_REFERENCE_DIR=<reference project> python tests/golden/make_golden.py
"""
import ctypes
import hashlib
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
from conftest import TRICLINIC, clustered_system, uniform_system  # noqa: E402

BETAS = [7.2462000846862793, 13.739999771118164, 20.736000061035156, 27.870000839233398]


def main():
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True, stdout=subprocess.DEVNULL)
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref.so"))
    D = ctypes.POINTER(ctypes.c_double)
    I = ctypes.POINTER(ctypes.c_int)
    lib.ref_pswf.argtypes = [ctypes.c_double, ctypes.c_int, D, D, D]
    lib.ref_legendre.argtypes = [ctypes.c_int, D, D]
    lib.ref_images.argtypes = [D, ctypes.c_double, ctypes.c_int, D, D, D, I, D, D, I, ctypes.c_long]
    lib.ref_images.restype = ctypes.c_long
    p = lambda a: a.ctypes.data_as(D)

    xs = np.linspace(0.0, 1.0, 41)
    pswf = []
    for b in BETAS:
        psi = np.zeros_like(xs)
        iv = np.zeros(4)
        lib.ref_pswf(b, len(xs), p(xs), p(psi), p(iv))
        pswf.append(dict(beta=b, x=xs.tolist(), psi=psi.tolist(), c0=iv[0], c1=iv[1], c2=iv[2], c4=iv[3]))
    json.dump(pswf, open(os.path.join(HERE, "pswf.json"), "w"), indent=1)

    leg = {}
    for n in (100, 200):
        x, w = np.zeros(n), np.zeros(n)
        lib.ref_legendre(n, p(x), p(w))
        leg[str(n)] = dict(x=x.tolist(), w=w.tolist())
    json.dump(leg, open(os.path.join(HERE, "legendre.json"), "w"))

    cases = []
    sysdefs = [
        ("cube_n20000_seed1", uniform_system(20000, 1), 4),
        ("cube_n3000_seed2_nz7", uniform_system(3000, 2), 7),
        ("triclinic_n4000_seed3", uniform_system(4000, 3, TRICLINIC), 4),
        ("triclinic_clustered_n4000_seed4", clustered_system(4000, 4, TRICLINIC), 4),
        ("swapped_axes_n2000_seed5", uniform_system(2000, 5, np.array([[0.8, 0.1, 0.0], [0, 1.3, 0.2], [0, 0, 1.0]])), 4),
    ]
    for name, (cell, pos, q), nz in sysdefs:
        avec = np.ascontiguousarray(cell.T).reshape(-1)
        pos = np.ascontiguousarray(pos)
        umat, qmat, xg, rc = np.zeros(9), np.zeros(9), np.zeros(3), np.zeros(1)
        mg = np.zeros(3, dtype=np.int32)
        cap = 50 * len(pos)
        idx = np.zeros(cap, dtype=np.int32)
        nimg = lib.ref_images(p(avec), float(nz), len(pos), p(pos), p(umat), p(qmat), mg.ctypes.data_as(I), p(xg),
                              p(rc), idx.ctypes.data_as(I), cap)
        idx = idx[:nimg]
        cases.append(dict(name=name, n=len(pos), nz=nz, n_images=int(nimg), umat=umat.tolist(), qmat=qmat.tolist(),
                          mgrid=mg.tolist(), xgrid0=xg.tolist(), rc=float(rc[0]),
                          img_idx_sha256=hashlib.sha256(idx.astype("<i4").tobytes()).hexdigest(),
                          img_idx_head=idx[:64].tolist()))
    json.dump(cases, open(os.path.join(HERE, "images.json"), "w"), indent=1)
    print("wrote pswf.json, legendre.json, images.json")


if __name__ == "__main__":
    main()
