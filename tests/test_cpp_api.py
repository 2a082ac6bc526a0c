"""The public C++ API (include/pdmk/periodic_dmk.hpp: PeriodicDMKTreeT<double>,
PeriodicDMKTreeT<float>, AutoPeriodicDMKTree, make_periodic_dmk_tree) compiled
into a C++ program against libpdmk_b200.so: the CPU test builds it, the GPU
test runs it (it checks the C++ API against the C ABI, see
tests/cpp/test_tree_api.cpp)."""
import os
import subprocess

import pytest

import periodicdmk_b200 as pd

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
EXE = os.path.join(ROOT, "periodicdmk_b200", "_build", "test_tree_api")


def _build():
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    lib = pd.library_path()
    cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), os.path.join(HERE, "cpp", "test_tree_api.cpp"),
           "-o", EXE, "-L", os.path.dirname(lib), "-lpdmk_b200", "-Wl,-rpath," + os.path.dirname(lib)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return EXE


def test_campaign_io_cpp(tmp_path):
    # include/pdmk/campaign_ref_io.hpp from C++ (host code only: runs on the CPU)
    if not os.path.exists(pd.library_path()):
        pytest.skip("libpdmk_b200.so not built")
    exe = str(tmp_path / "test_campaign_io")
    lib = pd.library_path()
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(HERE, "cpp", "test_campaign_io.cpp"), "-o", exe, "-L", os.path.dirname(lib),
                    "-lpdmk_b200", "-Wl,-rpath," + os.path.dirname(lib)], check=True, capture_output=True, text=True)
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=120)
    print(r.stdout)
    assert r.returncode == 0 and "0 failures" in r.stdout, r.stdout + r.stderr


def test_cpp_api_compiles_and_links():
    if not os.path.exists(pd.library_path()):
        pytest.skip("libpdmk_b200.so not built")
    assert os.path.exists(_build())


@pytest.mark.gpu
def test_cpp_api_matches_c_abi():
    exe = _build()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failures" in r.stdout
