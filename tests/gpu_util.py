"""Helpers shared by the GPU parity tests."""
import numpy as np

from single_svdlib import CooMatrix, CscMatrix, CsrMatrix, MaskedCSRMatrix

import matrices as M


def upload(kind, A, mask=None, dtype=np.float64):
    """The matrix as a device handle; dtype=np.float32 makes a T = f32 matrix."""
    v = lambda d: np.asarray(d, dtype=dtype)  # noqa: E731
    if kind == "csr":
        return CsrMatrix(A["nrows"], A["ncols"], A["indptr"], A["indices"], v(A["data"]))
    if kind == "csc":
        C = M.to_csc(A)
        return CscMatrix(C["nrows"], C["ncols"], C["indptr"], C["indices"], v(C["data"]))
    if kind == "coo":
        C = M.to_coo(A)
        return CooMatrix(C["nrows"], C["ncols"], C["row"], C["col"], v(C["data"]))
    if kind == "masked":
        parent = CsrMatrix(A["nrows"], A["ncols"], A["indptr"], A["indices"], v(A["data"]))
        return MaskedCSRMatrix(parent, mask)
    raise ValueError(kind)


def oracle_args(kind, A):
    if kind == "csc":
        return M.to_csc(A)
    if kind == "coo":
        return M.to_coo(A)
    return A


def assert_rows_parallel(X, Y, tol):
    """Row i of X equals row i of Y up to sign (unit rows)."""
    for i in range(X.shape[0]):
        a, b = X[i], Y[i]
        na, nb = np.linalg.norm(a), np.linalg.norm(b)
        if na == 0 or nb == 0:
            assert na == nb
            continue
        c = abs(a @ b) / (na * nb)
        assert abs(c - 1.0) < tol, (i, c)


def subspace_cos(U, V):
    """Cosines of the principal angles between the column spaces of U and V."""
    qu, _ = np.linalg.qr(U)
    qv, _ = np.linalg.qr(V)
    return np.linalg.svd(qu.T @ qv, compute_uv=False)
