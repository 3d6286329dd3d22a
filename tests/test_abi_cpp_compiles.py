"""The C++ adaptor header (include/hyteg_b200.hpp) and its test program compile and link against the
library on a machine without a GPU (the program itself runs in tests/test_gpu_cpp_abi.py)."""

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_adaptor_compiles_and_links(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    libdir = os.path.join(ROOT, "hyteg_b200")
    if not os.path.exists(os.path.join(libdir, "libhyteg_b200.so")):
        pytest.skip("library not built")
    subprocess.run([cxx, "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "gmg_apply.cpp"), "-L", libdir, "-lhyteg_b200",
                    f"-Wl,-rpath,{libdir}", "-o", str(tmp_path / "gmg_apply")], check=True)
    assert os.path.exists(tmp_path / "gmg_apply")
