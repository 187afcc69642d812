"""The rotations ritvec applies in SVDLIBC mode come from lanso's last Ritz
analysis (imtqlb, legacy.rs:961-1070) instead of a second QL pass (imtql2,
legacy.rs:1575-1692).  This compiles the host QL routines the library uses
(single-svdlib_b200/csrc/ql_host.h) into tests/ql_record_check.cpp and checks,
on random, graded and clustered tridiagonals and on the Lanczos T of real LAS2
runs (from the oracle), that the record is imtql2's bit for bit: the same
(i, c, s) list, the same converged eigenvalues and the same column order.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import matrices as M
import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "single-svdlib_b200", "csrc")
CUDA_INC = "/usr/local/cuda/include"


def lanczos_t(alf, bet):
    """(d, e) as lanso and ritvec build them from alpha and beta (reversed)."""
    j = len(alf) - 1
    d = np.asarray(alf, dtype=np.float64)[::-1].copy()
    e = np.zeros(j + 1)
    e[1:] = np.asarray(bet, dtype=np.float64)[1:j + 1][::-1]
    return d, e


def cases():
    rng = np.random.default_rng(5)
    out = []
    for n in (1, 2, 3, 5, 17, 64, 150):
        out.append((rng.standard_normal(n), np.r_[0.0, rng.standard_normal(n - 1)]))
    for n in (40, 120):  # graded, and clustered pairs as Lanczos ghosts make them
        out.append((np.geomspace(1e6, 1e-6, n), np.r_[0.0, np.geomspace(1e3, 1e-9, n - 1)]))
        base = np.repeat(rng.uniform(1, 10, n // 2), 2) + rng.standard_normal(n) * 1e-13
        out.append((base, np.r_[0.0, rng.standard_normal(n - 1) * 1e-3]))
    out.append((np.ones(30), np.r_[0.0, np.zeros(29)]))  # split everywhere
    for A, dims in ((M.poisson_rows(600, 300, 12, 3), 10), (M.uniform(200, 120, 0.1, 7), 6),
                    (M.lowrank_plus_noise(300, 150, 8, 1e-3, 2, density=0.3), 8)):
        r = O.las2("csr", A, dims, 0, seed=11, legacy=True)
        out.append(lanczos_t(r["alf"], r["bet"]))
    return out


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None or not os.path.exists(os.path.join(CUDA_INC, "cuda_runtime.h")):
        pytest.skip("needs g++ and the CUDA headers")
    exe = str(tmp_path_factory.mktemp("ql") / "ql_record_check")
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", CSRC, "-I", CUDA_INC,
                    os.path.join(ROOT, "tests", "ql_record_check.cpp"), "-o", exe], check=True)
    return exe


def test_imtqlb_record_is_imtql2(checker, tmp_path):
    path = tmp_path / "t.bin"
    with open(path, "wb") as f:
        for d, e in cases():
            n = len(d)
            f.write(np.int64(n).tobytes())
            f.write(np.asarray(d, dtype=np.float64).tobytes())
            f.write(np.asarray(e, dtype=np.float64).tobytes())
    res = subprocess.run([checker, str(path)], capture_output=True, text=True)
    assert res.returncode == 0, res.stdout + res.stderr
    ok, ncase, nrot = res.stdout.split()
    assert ok == "ok" and int(ncase) == len(cases()) and int(nrot) > 1000, res.stdout
