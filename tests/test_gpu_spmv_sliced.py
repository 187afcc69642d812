"""The column-sliced SpMV (csrc/spmv_sliced.cu) against FP64 products and the
gather kernel: svd_opa of A and A^T (src/lanczos/mod.rs:1551-1602) on
operators large enough to get the plan (more than 2^22 nonzeros, more than
one slice of 18,432 columns; the kernel is opt-in, SVDB_SPMV=sliced), with skewed row lengths (rows longer than a
slice, empty rows, rows inside one slice), FP64 values within 1e-13 and FP32
values (SVDB_MIXED) within 1e-6 of sum |a||x|; a LAS2 solve on the same
operator against the checker."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

import matrices as M
import oracle as O
from gpu_util import upload
from single_svdlib import _abi, legacy

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _sliced(monkeypatch):
    monkeypatch.setenv("SVDB_SPMV", "sliced")  # the kernel is opt-in


@pytest.fixture(scope="module")
def big():
    rng = np.random.default_rng(13)
    m, n = 300_000, 61_000
    lens = np.minimum(n, (rng.pareto(1.3, m) * 6 + 1).astype(np.int64))
    lens[:3] = [40_000, 25_000, 0]
    lens[10:20] = 0
    rows = np.repeat(np.arange(m), lens)
    cols = rng.integers(0, n, rows.size)
    S = sp.csr_matrix((rng.standard_normal(rows.size), (rows, cols)), shape=(m, n))
    S.sum_duplicates()
    S.sort_indices()
    assert S.nnz > (1 << 22)
    return M.from_scipy(S)


def info(h, transposed):
    ns, nr = C.c_int32(0), C.c_int32(0)
    assert _abi.lib().svdb_sliced_spmv_info(h.handle, int(transposed), C.byref(ns), C.byref(nr)) == 0
    return ns.value, nr.value


def opa_device(h, x, transposed, precision):
    import torch
    out = h.ncols() if transposed else h.nrows()
    dx = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    dy = torch.full((out,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = _abi.lib().svdb_opa_device(h.handle, dx.data_ptr(), dy.data_ptr(), int(transposed), precision, None)
    assert rc == 0, _abi.last_error()
    torch.cuda.synchronize()
    return dy.cpu().numpy()


@pytest.mark.parametrize("transposed", [False, True])
def test_sliced_products(big, transposed, monkeypatch):
    A = big
    S = M.to_scipy(A)
    h = upload("csr", A)
    rng = np.random.default_rng(3)
    x = rng.standard_normal(A["nrows"] if transposed else A["ncols"])
    want = (S.T @ x) if transposed else (S @ x)
    mag = (abs(S).T @ np.abs(x)) if transposed else (abs(S) @ np.abs(x))
    mag = np.maximum(mag, 1e-300)
    got = opa_device(h, x, transposed, 0)
    ns, nr = info(h, transposed)
    n_minor = A["nrows"] if transposed else A["ncols"]
    assert ns == (n_minor + 18431) // 18432 and nr >= 1
    assert np.max(np.abs(got - want) / mag) < 1e-13
    got32 = opa_device(h, x, transposed, 1)
    S32 = S.astype(np.float32).astype(np.float64)
    want32 = (S32.T @ x) if transposed else (S32 @ x)
    assert np.max(np.abs(got32 - want32) / mag) < 1e-13
    assert np.max(np.abs(got32 - want) / mag) < 1e-6
    # the gather kernel on a fresh handle gives the same product to rounding
    monkeypatch.setenv("SVDB_SPMV", "gather")
    h2 = upload("csr", A)
    g = opa_device(h2, x, transposed, 0)
    assert info(h2, transposed) == (0, 0)
    assert np.max(np.abs(g - got) / mag) < 1e-13


def test_sliced_deterministic_and_opb(big):
    A = big
    h = upload("csr", A)
    x = np.random.default_rng(4).standard_normal(A["ncols"])
    a, b = opa_device(h, x, False, 0), opa_device(h, x, False, 0)
    np.testing.assert_array_equal(a, b)
    S = M.to_scipy(A)
    want = S.T @ (S @ x)
    got = h.svd_opb(x)
    mag = np.maximum(abs(S).T @ (abs(S) @ np.abs(x)), 1e-300)
    assert np.max(np.abs(got - want) / mag) < 1e-12


def test_las2_on_a_sliced_operator(big):
    A = big
    got = legacy.svd_dim_seed(upload("csr", A), 4, 9)
    ref = O.las2("csr", A, 4, 0, seed=9, legacy=True)
    assert got.d == ref["d"] and got.diagnostics.lanczos_steps == ref["diagnostics"]["lanczos_steps"]
    np.testing.assert_allclose(got.s, ref["s"], rtol=1e-10)
