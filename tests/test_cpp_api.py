"""The header-only C++ API (include/nelson_b200/nelson.hpp).

CPU: the header and the C++ test program compile and link against the
library.  GPU: the program runs (host-loop LM / GN vs the device loop, fixed
nodes, cost reduction) and exits 0.
"""
import os
import shutil
import subprocess

import pytest

from nelson_b200 import build as nb_build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_api.cpp")


def _compile(out_dir):
    gxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    if gxx is None:
        pytest.skip("no C++ compiler")
    if not os.path.exists(nb_build.LIB):
        nb_build.build()
    exe = os.path.join(out_dir, "test_api")
    lib_dir = os.path.dirname(nb_build.LIB)
    cmd = [gxx, "-O2", "-std=c++17", "-Wall", "-Wextra", "-I" + os.path.join(ROOT, "include"), SRC,
           "-o", exe, "-L" + lib_dir, "-lnelson_b200", "-Wl,-rpath," + lib_dir,
           "-Wl,--allow-shlib-undefined"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "warning" not in r.stderr, r.stderr
    return exe


def test_cpp_api_compiles(tmp_path):
    assert os.path.exists(_compile(str(tmp_path)))


@pytest.mark.gpu
def test_cpp_api_runs(tmp_path):
    exe = _compile(str(tmp_path))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL OK" in r.stdout


def test_cpp_problem_file_readers(tmp_path):
    """The header's Problem / BALData readers (host code only, runs on CPU)."""
    gxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    if gxx is None:
        pytest.skip("no C++ compiler")
    exe = str(tmp_path / "test_loader")
    src = os.path.join(ROOT, "tests", "cpp", "test_loader.cpp")
    r = subprocess.run([gxx, "-O1", "-std=c++17", "-Wall", "-Wextra", "-I" + os.path.join(ROOT, "include"), src,
                        "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL OK" in r.stdout
