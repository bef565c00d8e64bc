"""The C ABI library loads without a GPU and exports every entry point that
include/hm.h declares; the oracle library builds and loads."""
import ctypes
import os
import re

import pytest

from conftest import PKG, ROOT

HDR = os.path.join(ROOT, "include", "hm.h")


def declared_symbols():
    src = open(HDR).read()
    return sorted(set(re.findall(r"HM_API\s+[\w\s\*]*?\b(hm_\w+)\s*\(", src)))


def test_header_declares_the_pipeline():
    syms = declared_symbols()
    for s in ["hm_generate_dataset", "hm_kdtree_build", "hm_structure_build", "hm_hmatrix_build",
              "hm_hmatvec", "hm_last_error"]:
        assert s in syms


def test_library_exports_every_declared_symbol():
    path = os.path.join(PKG, "libhmb200.so")
    if not os.path.exists(path):
        pytest.skip("libhmb200.so not built (run __graft_entry__.build())")
    lib = ctypes.CDLL(path)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, "not exported: %s" % missing


def test_version_and_error_string_without_gpu():
    path = os.path.join(PKG, "libhmb200.so")
    if not os.path.exists(path):
        pytest.skip("libhmb200.so not built")
    lib = ctypes.CDLL(path)
    lib.hm_version.restype = ctypes.c_char_p
    lib.hm_last_error.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.hm_version()
    # argument validation happens before any CUDA call
    lib.hm_kdtree_build.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
    out = ctypes.c_void_p()
    assert lib.hm_kdtree_build(None, 10, 2, 4, None, ctypes.byref(out)) == 1  # HM_ERR_INVALID
    assert b"NULL" in lib.hm_last_error()
    assert lib.hm_kdtree_build(ctypes.c_void_p(8), 10, 0, 4, None, ctypes.byref(out)) == 1
    assert out.value is None


def test_oracle_library_loads():
    import oracle

    assert oracle.tree_depth(8192, 32) == 8
    assert oracle.morton(1, 0) == 1 and oracle.morton(0, 1) == 2 and oracle.morton(3, 3) == 15


def test_refcompat_header_compiles(tmp_path):
    """The reference-name binding (include/hm_refcompat.h) is valid C++ over the
    C ABI, and the reference's main call sequence (tests/refcompat_main.cpp,
    run on a GPU by test_refcompat_gpu.py) compiles against it."""
    import subprocess

    src = tmp_path / "use.cpp"
    src.write_text('#include "hm_refcompat.h"\n'
                   'int main() { hmref::KDTree t; hmref::HMatrixStructure s; hmref::HMatrix h;\n'
                   '  (void)t; (void)s; (void)h; return 0; }\n')
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), "-I", cuda_inc,
                        os.path.join(ROOT, "tests", "refcompat_main.cpp")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_division_methods_validate_without_gpu():
    """hm_kdtree_build_div: an unknown DIVISION_METHOD is HM_ERR_INVALID and
    POWER_OF_TWO_ON_LEFT on a non-power-of-two n is HM_ERR_UNSUPPORTED, both
    before any CUDA call."""
    path = os.path.join(PKG, "libhmb200.so")
    if not os.path.exists(path):
        pytest.skip("libhmb200.so not built")
    lib = ctypes.CDLL(path)
    lib.hm_last_error.restype = ctypes.c_char_p
    P, I = ctypes.c_void_p, ctypes.c_int
    lib.hm_kdtree_build_div.argtypes = [P, I, I, I, I, P, ctypes.POINTER(P)]
    out = ctypes.c_void_p()
    assert lib.hm_kdtree_build_div(ctypes.c_void_p(8), 100, 2, 4, 7, None, ctypes.byref(out)) == 1
    assert b"division" in lib.hm_last_error()
    assert lib.hm_kdtree_build_div(ctypes.c_void_p(8), 100, 2, 4, 0, None, ctypes.byref(out)) == 4
    assert b"power-of-two" in lib.hm_last_error()
    assert out.value is None


def test_header_is_plain_c(tmp_path):
    import subprocess

    src = tmp_path / "use.c"
    src.write_text('#include "hm.h"\nint main(void) { hm_build_opts o; (void)o; return 0; }\n')
    r = subprocess.run(["gcc", "-std=c99", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_solver_and_file_entry_points_validate_without_gpu(tmp_path):
    """hm_cg_solve, hm_hmatrix_save and hm_hmatrix_load refuse null handles
    and bad sizes before any CUDA call."""
    path = os.path.join(PKG, "libhmb200.so")
    if not os.path.exists(path):
        pytest.skip("libhmb200.so not built")
    lib = ctypes.CDLL(path)
    lib.hm_last_error.restype = ctypes.c_char_p
    P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    lib.hm_cg_solve.argtypes = [P, I, P, I, P, I, D, I, I, P, P, P]
    lib.hm_hmatrix_save.argtypes = [P, ctypes.c_char_p]
    lib.hm_hmatrix_load.argtypes = [P, P, ctypes.c_char_p, P, ctypes.POINTER(P)]
    assert lib.hm_cg_solve(None, 1, None, 1, None, 1, 1e-6, 10, 4, None, None, None) == 1
    assert b"null matrix" in lib.hm_last_error()
    assert lib.hm_hmatrix_save(None, str(tmp_path / "x.hmb").encode()) == 1
    out = ctypes.c_void_p()
    assert lib.hm_hmatrix_load(None, None, b"x", None, ctypes.byref(out)) == 1
    assert out.value is None
    assert lib.hm_hmatrix_load(None, None, b"x", None, None) == 1


def test_check_and_schedule_entry_points_validate_without_gpu():
    """hm_hmatrix_check (the report of a device-side wait that gave up) and
    hm_schedule_set refuse null arguments before any CUDA call."""
    path = os.path.join(PKG, "libhmb200.so")
    if not os.path.exists(path):
        pytest.skip("libhmb200.so not built")
    lib = ctypes.CDLL(path)
    lib.hm_last_error.restype = ctypes.c_char_p
    P = ctypes.c_void_p
    lib.hm_hmatrix_check.argtypes = [P, P]
    lib.hm_schedule_set.argtypes = [P, ctypes.c_char_p, P]
    assert lib.hm_hmatrix_check(None, None) == 1
    assert b"null matrix" in lib.hm_last_error()
    assert lib.hm_schedule_set(None, b"mixed chunk_tiles=128 group_tiles=8 p1_ring=0 wide_tc=1 tc_chunk=32", None) == 1
    assert lib.hm_schedule_set(None, None, None) == 1


def test_python_wrappers_check_vector_shapes():
    """The C ABI trusts the sizes it is given; the Python wrappers check a
    block of vectors (float32 CUDA tensor, shape (n, nrhs)) before calling it."""
    import torch

    import hmatrix

    with pytest.raises(ValueError, match="shape"):
        hmatrix._check_vectors(torch.zeros((3, 100)), 100, "B")  # (nrhs, n) by mistake
    with pytest.raises(ValueError, match="shape"):
        hmatrix._check_vectors(torch.zeros((100, 0)), 100, "B")
    with pytest.raises(ValueError, match="float32 CUDA"):
        hmatrix._check_vectors(torch.zeros((100, 3)), 100, "B")  # a host tensor
    with pytest.raises(ValueError, match="float32 CUDA"):
        hmatrix._check_vectors(torch.zeros((100, 3), dtype=torch.float64), 100, "B")
