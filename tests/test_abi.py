"""The C ABI: every symbol of include/svdb200.h is exported, and the
host-side argument handling of svd_las2 (no GPU needed)."""
import os
import re

import pytest

from single_svdlib import Las2Error, _abi
from single_svdlib.lanczos import las2_plan

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "svdb200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(svdb_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_functions():
    names = declared_functions()
    assert "svdb_las2" in names and "svdb_randomized_svd" in names and "svdb_masked_new" in names


def test_library_exports_every_declared_symbol():
    L = _abi.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    assert set(declared_functions()) == set(_abi.SIGNATURES)


def test_status_codes_are_svdliberror_variants():
    text = open(HEADER).read()
    codes = dict(re.findall(r"(SVDB_ERR_[A-Z0-9]+)\s*=\s*(\d+)", text))
    assert codes["SVDB_ERR_IMTQLB"] == "1" and codes["SVDB_ERR_STARTV"] == "2"
    assert codes["SVDB_ERR_STPONE"] == "3" and codes["SVDB_ERR_IMTQL2"] == "4" and codes["SVDB_ERR_LAS2"] == "5"


def test_las2_plan_clamps_like_svd_las2():  # src/lanczos/mod.rs:121-141
    assert las2_plan(100, 50, 10, 0, 0)[:2] == (50, 50)
    assert las2_plan(100, 50, 10, 80, 0)[:2] == (50, 50)
    assert las2_plan(100, 50, 10, 10, 5)[:2] == (10, 10)
    assert las2_plan(100, 50, 10, 10, 30)[:2] == (10, 30)
    assert las2_plan(100, 50, 10, 10, 500)[:2] == (10, 50)


def test_las2_plan_transpose_rule():  # mod.rs:143: ncols >= 1.2 nrows
    assert las2_plan(10, 12, 5)[2] is True
    assert las2_plan(10, 11, 5)[2] is False
    assert las2_plan(5000, 2000, 100000)[2] is False


def test_las2_plan_sparsity_branches():  # mod.rs:1276-1300
    assert las2_plan(5000, 2000, 99567)[3] == 2
    assert las2_plan(100, 100, 5000)[3] == 0
    assert las2_plan(100, 100, 500)[3] == 1
    assert las2_plan(1000, 1000, 500)[3] == 3


def test_las2_plan_insufficient_dimensions():  # mod.rs:134-138
    with pytest.raises(Las2Error, match="insufficient dimensions: 1"):
        las2_plan(1, 5, 3)
