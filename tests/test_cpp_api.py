"""The header-only C++ API (include/nelson_b200/nelson.hpp).

CPU: the header and the C++ test programs compile and link against the
library.  GPU: test_api runs (host-loop LM / GN vs the device loop, fixed
nodes, cost reduction, the envelope solver and camera orders, the
ScanAlignSection single section reaching chi2 < 1e-12) and exits 0;
test_section_edges (nvcc) subclasses DeviceEdgeSection with CUDA edge
kernels and reaches chi2 < 1e-12 and the true parameters; test_solver_concept drives the
reference-shaped LevenbergMarquardt / GaussNewton loops (the calls of
nelson/LevenbergMarquardt.hpp:36-146 on the Solver and problem concepts) with
a host-assembled problem (the reference's 5 x 2D / 3 x 3D fixture, final
chi2 < 1e-12) and with a BASection read from a BAL file, whose per-sub-
iteration trace must match the FP64 oracle's (1e-9 FP64, 1e-6 mixed).
"""
import os
import shutil
import subprocess

import pytest

from nelson_b200 import build as nb_build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _compile(out_dir, name="test_api"):
    gxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    if gxx is None:
        pytest.skip("no C++ compiler")
    if not os.path.exists(nb_build.LIB):
        nb_build.build()
    exe = os.path.join(out_dir, name)
    lib_dir = os.path.dirname(nb_build.LIB)
    src = os.path.join(ROOT, "tests", "cpp", name + ".cpp")
    cmd = [gxx, "-O2", "-std=c++17", "-Wall", "-Wextra", "-I" + os.path.join(ROOT, "include"), src,
           "-o", exe, "-L" + lib_dir, "-lnelson_b200", "-Wl,-rpath," + lib_dir,
           "-Wl,--allow-shlib-undefined"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "warning" not in r.stderr, r.stderr
    return exe


def _compile_cu(out_dir, name):
    """An nvcc-compiled C++ test (user edges as CUDA kernels), sm_100a."""
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("no nvcc")
    if not os.path.exists(nb_build.LIB):
        nb_build.build()
    exe = os.path.join(out_dir, name)
    lib_dir = os.path.dirname(nb_build.LIB)
    src = os.path.join(ROOT, "tests", "cpp", name + ".cu")
    cmd = [nvcc, "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-I" + os.path.join(ROOT, "include"),
           src, "-o", exe, "-L" + lib_dir, "-lnelson_b200", "-Xlinker", "-rpath," + lib_dir,
           "-Xlinker", "--allow-shlib-undefined"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_section_edges_compiles(tmp_path):
    assert os.path.exists(_compile_cu(str(tmp_path), "test_section_edges"))


@pytest.mark.gpu
def test_section_edges_runs(tmp_path):
    """DeviceEdgeSection subclassed with CUDA edge kernels: LM and GN, natural
    and AMD order, reach chi2 < 1e-12 and the true parameters."""
    exe = _compile_cu(str(tmp_path), "test_section_edges")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL OK" in r.stdout


def test_cpp_api_compiles(tmp_path):
    assert os.path.exists(_compile(str(tmp_path)))
    assert os.path.exists(_compile(str(tmp_path), "test_solver_concept"))


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


@pytest.mark.gpu
def test_reference_concept_loops(tmp_path, oracle_lib):
    import numpy as np

    from nelson_b200 import problems as P
    exe = _compile(str(tmp_path), "test_solver_concept")
    p = P.make_config(1, 0.05)  # 10 cameras x 9, 2,500 points
    p.obs = p.obs - np.array([p.cx, p.cy])
    p.cx = p.cy = 0.0
    bal = str(tmp_path / "scene.bal")
    P.save_bal(bal, p)
    its = 8
    r = subprocess.run([exe, bal, str(its)], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL OK" in r.stdout
    o = oracle_lib.Oracle.from_ba(P.load_bal(bal))
    _, tr_o, _, _ = o.lm_solve(oracle_lib.LMSettings(maxNumIt=its))
    for prec, tol in ((0, 1e-9), (1, 1e-6)):
        rows = [ln.split()[2:] for ln in r.stdout.splitlines() if ln.startswith(f"TRACE {prec} ")]
        tr = np.array([[float(x) for x in row] for row in rows])
        assert len(tr) == len(tr_o), (prec, len(tr), len(tr_o))
        for k in range(len(tr)):
            if tr_o[k, 2] < 0:
                continue
            assert abs(tr[k, 2] - tr_o[k, 2]) <= tol * tr_o[k, 2], (prec, k, tr[k], tr_o[k])
            if tr_o[k, 3] != 0:
                assert tr[k, 3] == pytest.approx(tr_o[k, 3], rel=1e-6), (prec, k)
