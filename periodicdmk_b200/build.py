"""Build libpdmk_b200.so in-tree (sm_100a).

    python -m periodicdmk_b200.build          # incremental
    python -m periodicdmk_b200.build --clean  # rebuild everything

CUDA sources are compiled by nvcc for ``-gencode arch=compute_100a,code=sm_100a``;
host C++ by g++.  cudart is linked statically, so the library does not depend
on whichever CUDA runtime the host process (e.g. torch) loaded; cuFFT is linked
dynamically (libcufft from the CUDA toolkit's lib64, found through an rpath).
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB_DIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIB_DIR, "libpdmk_b200.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INCLUDES = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
CXX = "g++"


def _sources():
    out = []
    for sub in ("host", "device", "api"):
        d = os.path.join(CSRC, sub)
        for f in sorted(os.listdir(d)):
            if f.endswith((".cu", ".cpp")):
                out.append(os.path.join(d, f))
    return out


def _headers():
    hs = []
    for base in (CSRC, os.path.join(ROOT, "include")):
        for dp, _, fs in os.walk(base):
            hs += [os.path.join(dp, f) for f in fs if f.endswith((".h", ".hpp", ".cuh"))]
    return hs


def _obj(src):
    rel = os.path.relpath(src, CSRC).replace(os.sep, "_")
    return os.path.join(BUILD, rel + ".o")


def _compile(src):
    obj = _obj(src)
    if src.endswith(".cu"):
        cmd = [NVCC] + ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                                "--expt-relaxed-constexpr"] + INCLUDES + ["-c", src, "-o", obj]
    else:
        cmd = [CXX, "-O3", "-std=c++17", "-fPIC", "-I", os.path.join(CUDA_HOME, "include")] + INCLUDES + \
              ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return obj


def build(clean=False, verbose=True):
    if clean and os.path.isdir(BUILD):
        shutil.rmtree(BUILD)
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    srcs = _sources()
    hdr_mtime = max(os.path.getmtime(h) for h in _headers())
    todo = [s for s in srcs if not os.path.exists(_obj(s)) or
            os.path.getmtime(_obj(s)) < max(os.path.getmtime(s), hdr_mtime)]
    if todo:
        if verbose:
            print("compiling %d sources" % len(todo), file=sys.stderr)
        with cf.ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            list(ex.map(_compile, todo))
    objs = [_obj(s) for s in srcs]
    if todo or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + \
              ["-cudart", "static", "-L", os.path.join(CUDA_HOME, "lib64"), "-lcufft",
               "-Xlinker", "-rpath=" + os.path.join(CUDA_HOME, "lib64"), "-lpthread", "-ldl", "-lrt"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
        if verbose:
            print("linked", LIB, file=sys.stderr)
    return LIB


if __name__ == "__main__":
    build(clean="--clean" in sys.argv)
