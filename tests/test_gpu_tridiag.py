"""The tridiagonal QL recurrences run on the device (svdb_tridiag_device, one
GPU thread, FP64, unfused) against the checker's host restatements
(oracle/svd_oracle.cpp): imtqlb of SVDLIBC and as written
(src/legacy.rs:955-1070, src/lanczos/mod.rs:428-584) and imtql2
(src/lanczos/mod.rs:901-1028) must agree bit for bit on the tridiagonals of
test_ql_record.py (random, graded, clustered, split, and the Lanczos T of three
LAS2 runs), imtql2's eigenvectors rebuilt from the device's rotation record.
The time of each side on the Lanczos T of the 5,000 x 2,000 LAS2 workload is
printed (the solver keeps the faster host form).
"""
import ctypes as C
import time

import numpy as np
import pytest

import matrices as M
import oracle as O
from single_svdlib import _abi
from test_ql_record import cases, lanczos_t

pytestmark = pytest.mark.gpu


def device(routine, d, e, max_it=30, rot_cap=None):
    n = len(d)
    d = np.ascontiguousarray(d, dtype=np.float64).copy()
    e = np.ascontiguousarray(e, dtype=np.float64).copy()
    bnd = np.zeros(n)
    perm = np.zeros(n, np.int32)
    cap = (60 * n * n + 16) if rot_cap is None else rot_cap
    ri, rc, rs = np.zeros(cap, np.int32), np.zeros(cap), np.zeros(cap)
    nrot, warned, ms = C.c_uint64(0), C.c_int(0), C.c_double(0)
    rc_ = _abi.lib().svdb_tridiag_device(routine, n, d.ctypes.data, e.ctypes.data, bnd.ctypes.data, ri.ctypes.data,
                                         rc.ctypes.data, rs.ctypes.data, cap, C.byref(nrot), perm.ctypes.data, max_it,
                                         C.byref(warned), C.byref(ms))
    k = min(nrot.value, cap)
    return {"status": rc_, "d": d, "e": e, "bnd": bnd, "perm": perm, "rot": (ri[:k], rc[:k], rs[:k]),
            "nrot": nrot.value, "warned": warned.value, "ms": ms.value}


def apply_rotations(n, rot, perm):
    """imtql2's z (identity start), from its rotation record, then its column order."""
    z = np.eye(n)
    for i, c, s in zip(*rot):
        f = z[:, i + 1].copy()
        z[:, i + 1] = s * z[:, i] + c * f
        z[:, i] = c * z[:, i] - s * f
    return z[:, perm]


@pytest.mark.parametrize("legacy", [True, False])
def test_imtqlb_bit_equal_to_checker(legacy):
    for k, (d, e) in enumerate(cases()):
        got = device(0 if legacy else 1, d, e, max_it=30 if legacy else 100)
        try:
            rd, rb = O.imtqlb(d, e, legacy=legacy, max_it=100)
        except O.OracleError as x:
            assert got["status"] == 1 and x.kind == "ImtqlbError", k
            continue
        assert got["status"] == 0, (k, _abi.last_error())
        assert np.array_equal(got["d"], rd), k
        assert np.array_equal(got["bnd"], rb), k


@pytest.mark.parametrize("legacy", [True, False])
def test_imtql2_bit_equal_to_checker(legacy):
    total = 0
    for k, (d, e) in enumerate(cases()):
        n = len(d)
        got = device(2 if legacy else 3, d, e, max_it=30 if legacy else 50)
        try:
            rd, rz = O.imtql2(d, e, legacy=legacy, max_it=30 if legacy else 50)
        except O.OracleError as x:
            assert got["status"] == 4 and x.kind == "Imtql2Error", k
            continue
        assert got["status"] == 0, (k, _abi.last_error())
        assert got["nrot"] == len(got["rot"][0])
        total += got["nrot"]
        assert np.array_equal(got["d"], rd), k
        # the checker's z is row-major n x n with eigenvector j in column j
        assert np.array_equal(apply_rotations(n, got["rot"], got["perm"]), rz), k
    assert total > 1000


def test_error_paths_and_arguments():
    d, e = cases()[5]
    got = device(2, d, e, max_it=1)  # an iteration cap of 1 cannot converge on this T
    assert got["status"] == 4 and "imtql2" in _abi.last_error()
    assert device(9, d, e)["status"] == 10


def test_device_against_host_time():
    """The Lanczos T of the 5,000 x 2,000 LAS2 workload (js = 192)."""
    A = M.poisson_rows(5000, 2000, 20, 42)
    r = O.las2("csr", A, 10, 0, seed=42, legacy=True)
    d, e = lanczos_t(r["alf"], r["bet"])
    got = device(0, d, e)
    assert got["status"] == 0
    reps = 5
    t0 = time.perf_counter()
    for _ in range(reps):
        rd, rb = O.imtqlb(d, e, legacy=True)
    host_ms = (time.perf_counter() - t0) / reps * 1e3
    assert np.array_equal(got["d"], rd) and np.array_equal(got["bnd"], rb)
    print(f"imtqlb SVDLIBC, n={len(d)}, {got['nrot']} rotations: device {got['ms']:.3f} ms, host {host_ms:.3f} ms")
