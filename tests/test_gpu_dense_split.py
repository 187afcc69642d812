"""The dense-column split of the FP32 SpMM (csrc/dense_split.cu) against the
checker's products and the gather path.

Matrices with a few hundred columns of density above the 8 % threshold (the
split takes them to the tensor cores as a 3xTF32 GEMM) plus a sparse rest.
The products A X and A^T Y of the split must match the FP64 checker within
an FP32 accumulation bound (1e-5 of each output entry's magnitude,
sum |a||x|); randomized_svd under SVDB_MIXED must match the FP64 checker
within 1e-6 (sigma) with the split on and off.  Shapes cover a partial last
row tile, dense-column counts that are not a multiple of the 128-row tile,
l from 1 to 64, and a masked view.
"""
import numpy as np
import pytest

import matrices as M
import oracle as O
from gpu_util import upload
from single_svdlib import MaskedCSRMatrix, _abi, randomized
from single_svdlib.randomized import PowerIterationNormalizer as PIN

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _split_on(monkeypatch):
    monkeypatch.setenv("SVDB_DENSE_SPLIT", "1")  # the split is opt-in


def dense_cols_matrix(m, n, nd, seed):
    """nd columns with densities uniform in (0.1, 0.4), the others at 0.004."""
    return M.dense_columns(m, n, nd, seed)


def device_product(h, X, transpose):
    """svdb_multiply_with_dense_device under SVDB_MIXED (FP32 in and out)."""
    import torch
    rows = h.ncols() if transpose else h.nrows()
    dx = torch.from_numpy(np.ascontiguousarray(X, dtype=np.float32)).cuda()
    dy = torch.full((rows, X.shape[1]), float("nan"), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    rc = _abi.lib().svdb_multiply_with_dense_device(h.handle, dx.data_ptr(), X.shape[1], dy.data_ptr(),
                                                    int(transpose), 1, None)
    assert rc == 0, _abi.last_error()
    torch.cuda.synchronize()
    return dy.cpu().numpy().astype(np.float64)


def split_info(h):
    import ctypes as C
    nd, nnz = C.c_uint64(0), C.c_uint64(0)
    assert _abi.lib().svdb_dense_split_info(h.handle, C.byref(nd), C.byref(nnz)) == 0
    return nd.value, nnz.value


def check_product(A, got, X, transpose):
    S = M.to_scipy(A)
    X32 = X.astype(np.float32).astype(np.float64)
    want = (S.T @ X32) if transpose else (S @ X32)
    mag = (abs(S).T @ np.abs(X32)) if transpose else (abs(S) @ np.abs(X32))
    err = np.abs(got - want) / np.maximum(mag, 1e-300)
    assert np.all(np.isfinite(got))
    assert err.max() < 1e-5, err.max()


@pytest.mark.parametrize("m,n,nd,l", [(3000, 1500, 300, 60), (1111, 700, 129, 64), (2048, 900, 256, 1),
                                      (5003, 2100, 700, 17)])
def test_products_match_checker(m, n, nd, l, monkeypatch):
    A = dense_cols_matrix(m, n, nd, 7 + l)
    h = upload("csr", A)
    rng = np.random.default_rng(l)
    for transpose in (False, True):
        X = rng.standard_normal((m if transpose else n, l))
        monkeypatch.setenv("SVDB_DENSE_SPLIT", "1")
        split = device_product(h, X, transpose)
        nd_used, dense_nnz = split_info(h)
        assert nd_used == nd and 0 < dense_nnz < len(A["data"])
        check_product(A, split, X, transpose)
        monkeypatch.setenv("SVDB_DENSE_SPLIT", "0")
        gather = device_product(h, X, transpose)
        check_product(A, gather, X, transpose)


def test_masked_view_products():
    A = dense_cols_matrix(2500, 1200, 260, 3)
    mask = (np.random.default_rng(4).random(1200) < 0.8).astype(np.uint8)
    mv = MaskedCSRMatrix(upload("csr", A), mask)
    keep = np.flatnonzero(mask)
    Am = M.from_scipy(M.to_scipy(A)[:, keep])
    rng = np.random.default_rng(5)
    for transpose in (False, True):
        X = rng.standard_normal((2500 if transpose else len(keep), 40))
        check_product(Am, device_product(mv, X, transpose), X, transpose)


@pytest.mark.parametrize("split", ["1", "0"])
def test_randomized_mixed_matches_f64_checker(split, monkeypatch):
    monkeypatch.setenv("SVDB_DENSE_SPLIT", split)
    A = dense_cols_matrix(6000, 2500, 400, 11)
    rank, over, q, seed = 20, 10, 3, 5
    ref = O.randomized(A, rank, over, q, "QR", omega=O.omega_stream(seed, 2500, rank + over))
    got = randomized.randomized_svd(upload("csr", A), rank, over, q, PIN.QR, False, seed, False, precision="mixed")
    err = np.max(np.abs(got.s - ref["s"]) / ref["s"])
    assert err < 1e-6, err


def test_split_is_deterministic():
    A = dense_cols_matrix(3000, 1500, 300, 21)
    h = upload("csr", A)
    X = np.random.default_rng(2).standard_normal((1500, 60))
    a = device_product(h, X, False)
    b = device_product(h, X, False)
    np.testing.assert_array_equal(a, b)
    Y = np.random.default_rng(3).standard_normal((3000, 60))
    np.testing.assert_array_equal(device_product(h, Y, True), device_product(h, Y, True))
