"""Seeded synthetic sparse matrices for the tests (numpy PCG64 generators).

Each generator returns a dict with nrows, ncols, indptr, indices, data (CSR,
column indices ascending within a row), the layout the oracle and the
library both take.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def from_scipy(m) -> dict:
    m = sp.csr_matrix(m)
    m.sort_indices()
    return {"nrows": m.shape[0], "ncols": m.shape[1], "indptr": m.indptr.astype(np.int64),
            "indices": m.indices.astype(np.int64), "data": m.data.astype(np.float64)}


def to_scipy(A: dict):
    return sp.csr_matrix((A["data"], A["indices"], A["indptr"]), shape=(A["nrows"], A["ncols"]))


def to_csc(A: dict) -> dict:
    c = to_scipy(A).tocsc()
    c.sort_indices()
    return {"nrows": A["nrows"], "ncols": A["ncols"], "indptr": c.indptr.astype(np.int64),
            "indices": c.indices.astype(np.int64), "data": c.data.astype(np.float64)}


def to_coo(A: dict) -> dict:
    c = to_scipy(A).tocoo()
    return {"nrows": A["nrows"], "ncols": A["ncols"], "row": c.row.astype(np.int64), "col": c.col.astype(np.int64),
            "data": c.data.astype(np.float64)}


def dense(M) -> dict:
    return from_scipy(sp.csr_matrix(np.asarray(M, dtype=np.float64)))


def uniform(m, n, density, seed, low=-10.0, high=10.0) -> dict:
    """Distinct uniform positions, values U(low, high) (the crate's create_sparse_matrix shape,
    src/lib.rs:22-60, drawn with numpy instead of StdRng)."""
    rng = np.random.default_rng(seed)
    nnz = max(1, int(round(m * n * density)))
    flat = rng.choice(m * n, size=nnz, replace=False)
    r, c = np.divmod(flat, n)
    v = rng.uniform(low, high, nnz)
    return from_scipy(sp.csr_matrix((v, (r, c)), shape=(m, n)))


def poisson_rows(m, n, lam, seed, value_dist="uniform01") -> dict:
    """Per row Poisson(lam) distinct columns uniform in [0, n); values U(0,1)
    (the LAS2 f64 workload: 5000 x 2000, lam = 20, seed 42)."""
    rng = np.random.default_rng(seed)
    k = np.minimum(rng.poisson(lam, m), n)
    indptr = np.zeros(m + 1, np.int64)
    indptr[1:] = np.cumsum(k)
    idx = np.empty(indptr[-1], np.int64)
    for i in range(m):
        idx[indptr[i]:indptr[i + 1]] = np.sort(rng.choice(n, k[i], replace=False))
    val = rng.random(indptr[-1]) if value_dist == "uniform01" else rng.standard_normal(indptr[-1])
    return {"nrows": m, "ncols": n, "indptr": indptr, "indices": idx, "data": val}


def lowrank_plus_noise(m, n, rank, noise, seed, density=1.0) -> dict:
    rng = np.random.default_rng(seed)
    U = rng.standard_normal((m, rank))
    V = rng.standard_normal((n, rank))
    s = np.geomspace(100.0, 1.0, rank)
    M = (U * s) @ V.T / np.sqrt(m * n) * 10 + noise * rng.standard_normal((m, n))
    if density < 1.0:
        M[rng.random((m, n)) > density] = 0.0
    return dense(M)


def omega(n, l, seed) -> np.ndarray:
    return np.random.default_rng(seed).standard_normal((n, l))
