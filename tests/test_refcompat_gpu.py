"""The reference's pipeline through include/hm_refcompat.h, executed.

tests/refcompat_main.cpp is the reference's main call sequence
(src/main.cu:52-173: generateDataset -> allocateKDTree/constructKDTree ->
constructHMatrixStructure -> generateHMatrixFromStruct -> HMatrixVecMult with
FP64 vectors) written against the shim header and linked with -lhmb200, the
way a reference maintainer would switch.  This test compiles it with g++, runs
it, and checks what it wrote against the CPU oracle: the KD-tree permutation
and leaf offsets bit for bit, the FP64-vector product against a dense FP64
product, and the division-method handling.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG, ROOT

pytestmark = pytest.mark.gpu

CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _compile(tmp_path):
    exe = tmp_path / "refcompat_main"
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "refcompat_main.cpp"), "-o", str(exe), "-L", PKG, "-lhmb200",
           "-Wl,-rpath," + PKG, "-L", os.path.join(CUDA, "lib64"), "-lcudart", "-Wl,-rpath," + os.path.join(CUDA, "lib64")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def _read(path):
    buf = open(path, "rb").read()
    n, d, nrhs, depth, st_pow2 = np.frombuffer(buf, np.int32, 5, 0)
    off = 20

    def take(dt, cnt):
        nonlocal off
        a = np.frombuffer(buf, dt, cnt, off).copy()
        off += a.nbytes
        return a

    out = dict(n=int(n), d=int(d), nrhs=int(nrhs), depth=int(depth), status_pow2=int(st_pow2))
    out["points"] = take(np.float64, n * d)
    out["perm"] = take(np.int32, n)
    out["offsets"] = take(np.int32, (1 << depth) + 1)
    out["X"] = take(np.float64, n * nrhs).reshape(nrhs, n)
    out["Y"] = take(np.float64, n * nrhs).reshape(nrhs, n)
    assert off == len(buf)
    return out


def test_reference_main_through_the_shim(tmp_path):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import oracle

    exe = _compile(tmp_path)
    n, d, b, nrhs, tol = 8192, 2, 32, 3, 1e-6  # C1: the reference's default 2-D case
    outf = tmp_path / "out.bin"
    r = subprocess.run([str(exe), str(n), str(d), str(b), str(nrhs), str(tol), str(outf)], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ok" in r.stdout
    o = _read(outf)
    assert o["status_pow2"] == 4  # POWER_OF_TWO_ON_LEFT on 8191 points: HM_ERR_UNSUPPORTED
    ref = oracle.kdtree(o["points"], n, d, b)
    assert o["depth"] == ref["depth"]
    assert np.array_equal(o["perm"], ref["perm"])
    assert np.array_equal(o["offsets"], ref["offsets"])
    # the FP64-vector product (tree order) against a dense FP64 product on every
    # row; exp(-r/0.1), the reference's 2-D kernel (hm_build_opts_default)
    rows = np.arange(n, dtype=np.int32)
    Yref = oracle.dense_rows_matvec(o["points"], n, d, o["perm"], oracle.K_EXP, 0.1, 0.0, rows, o["X"])
    err = np.linalg.norm(o["Y"] - Yref) / np.linalg.norm(Yref)
    assert err < 1e-5, err
