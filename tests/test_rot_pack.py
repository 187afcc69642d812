"""The packed rotation lists of ritvec's device rotation kernel
(single-svdlib_b200/csrc/rot_pack.h), compiled with g++ into
tests/rot_pack_check.cpp: segment tiling and contents, the segment schedule
against the sequential loop of imtql2's vector accumulation (bit for bit),
piecewise packing, and refused indices.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "single-svdlib_b200", "csrc")
CUDA_INC = "/usr/local/cuda/include"


def test_rot_pack_contract(tmp_path):
    cxx = shutil.which("g++")
    if cxx is None or not os.path.exists(os.path.join(CUDA_INC, "cuda_runtime.h")):
        pytest.skip("needs g++ and the CUDA headers")
    exe = str(tmp_path / "rot_pack_check")
    subprocess.run([cxx, "-O2", "-std=c++17", "-ffp-contract=off", "-I", CSRC, "-I", CUDA_INC,
                    os.path.join(ROOT, "tests", "rot_pack_check.cpp"), "-o", exe], check=True)
    res = subprocess.run([exe], capture_output=True, text=True)
    assert res.returncode == 0, res.stdout + res.stderr
    ok, lists, nrot = res.stdout.split()
    assert ok == "ok" and int(lists) == 200 and int(nrot) > 100000, res.stdout
