"""The C-ABI library loads and exports every entry point include/nelson_b200.h
declares (no compute without a GPU)."""
import ctypes
import os
import re

import pytest

from nelson_b200 import build as nb_build
from nelson_b200 import native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "nelson_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(nl_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    nb_build.build()
    return ctypes.CDLL(nb_build.LIB)


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "nl_lm_solve" in syms and "nl_compute_increment" in syms and "nl_solver_create" in syms
    assert len(syms) >= 35


def test_library_exports_every_declared_symbol(lib):
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_exports():
    assert set(native.EXPORTS) <= set(declared_symbols())


def test_version_and_status_strings(lib):
    lib.nl_version.restype = ctypes.c_char_p
    lib.nl_status_string.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.nl_version()
    assert lib.nl_status_string(5) == b"not positive definite"


def test_bad_descriptors_rejected_without_device(lib):
    # argument validation happens before any CUDA call
    desc = native.ProblemDesc(bc=7, nc_var=1, nc_fix=0, np_var=1, np_fix=0, precision=0, f=500, cx=0, cy=0,
                              refine_sweeps=-1, device=0)
    h = ctypes.c_void_p()
    L = native.load()
    assert L.nl_create(ctypes.byref(desc), ctypes.byref(h)) == 1  # NL_ERR_ARG
    assert L.nl_create(None, ctypes.byref(h)) == 1


def test_header_is_c99_and_links(tmp_path):
    """include/nelson_b200.h is plain C (a cgo / JNI / ctypes binder includes
    it from C): a C99 program that takes the address of every declared entry
    point compiles with -pedantic -Werror and links against the library."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    nb_build.build()
    syms = declared_symbols()
    src = tmp_path / "abi.c"
    body = "\n".join(f"  (entry_point)&{s}," for s in syms)
    src.write_text('#include "nelson_b200.h"\n#include <stdio.h>\n'
                   "typedef void (*entry_point)(void);\n"
                   f"static const entry_point entry_points[] = {{\n{body}\n}};\n"
                   "int main(void) {\n  printf(\"%d\\n\", (int)(sizeof entry_points / sizeof entry_points[0]));\n"
                   "  return 0;\n}\n")
    exe = tmp_path / "abi"
    lib_dir = os.path.dirname(nb_build.LIB)
    r = subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror",
                        "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe), "-L" + lib_dir,
                        "-lnelson_b200", "-Wl,-rpath," + lib_dir, "-Wl,--allow-shlib-undefined"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert len(syms) > 80
