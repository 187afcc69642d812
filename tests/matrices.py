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


def count_like(m=100_000, n=30_000, seed=2024):
    """The randomized-SVD workload: a seeded count-like CSR.  Column rates
    lambda_j ~ Gamma(0.5, 2); row lengths ~ LogNormal(ln 600, 0.5), capped at n;
    columns drawn proportional to lambda_j with replacement and merged per row
    (the realised nnz is what the caller reports); values log1p(Poisson(lambda_j) + 1).
    Returns (indptr int64, cols int64, vals f64)."""
    rng = np.random.default_rng(seed)
    lam = rng.gamma(0.5, 2.0, n)
    k = np.clip(np.rint(rng.lognormal(np.log(600.0), 0.5, m)), 1, n).astype(np.int64)
    cdf = np.cumsum(lam / lam.sum())
    cdf[-1] = 1.0
    rows = np.repeat(np.arange(m, dtype=np.int64), k)
    cols = np.searchsorted(cdf, rng.random(rows.size), side="right").astype(np.int64)
    np.minimum(cols, n - 1, out=cols)
    keys = rows * n + cols
    keys.sort()
    keep = np.ones(keys.size, dtype=bool)
    keep[1:] = keys[1:] != keys[:-1]
    rows, cols = np.divmod(keys[keep], n)
    del keys, keep
    indptr = np.zeros(m + 1, np.int64)
    np.cumsum(np.bincount(rows, minlength=m), out=indptr[1:])
    vals = np.log1p(rng.poisson(lam[cols]) + 1.0)
    return indptr, cols, vals


def zipf_planted_device(torch, m=1_000_000, n=200_000, seed=3):
    """The large LAS2 workload, generated on the device (torch CUDA generator):
    row lengths Zipf(1.85) on [20, 20000] (numpy seed), columns uniform with
    duplicates merged, values N(0,1) plus a planted rank-20 signal
    sum_r s_r u_i v_j (unit u, v; s geometric 100..1, scaled by 1/density).
    Returns (indptr int64, cols int32, vals f64) as CUDA tensors."""
    rng = np.random.default_rng(seed)
    ks = np.arange(20, 20001)
    p = ks.astype(np.float64) ** -1.85
    p /= p.sum()
    rowlen = torch.from_numpy(rng.choice(ks, size=m, p=p)).cuda()
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    nnz0 = int(rowlen.sum())
    keys = torch.repeat_interleave(torch.arange(m, device="cuda", dtype=torch.int64), rowlen) * n
    keys += torch.randint(0, n, (nnz0,), device="cuda", generator=g, dtype=torch.int64)
    keys = torch.unique_consecutive(torch.sort(keys).values)
    rows = keys // n
    cols = (keys - rows * n).to(torch.int32)
    del keys
    nnz = rows.numel()
    indptr = torch.zeros(m + 1, dtype=torch.int64, device="cuda")
    indptr[1:] = torch.cumsum(torch.bincount(rows, minlength=m), 0)
    vals = torch.randn(nnz, dtype=torch.float64, device="cuda", generator=g)
    r = 20
    u = torch.randn(m, r, dtype=torch.float64, device="cuda", generator=g)
    v = torch.randn(n, r, dtype=torch.float64, device="cuda", generator=g)
    u /= u.norm(dim=0)
    v /= v.norm(dim=0)
    sig = torch.logspace(2, 0, r, dtype=torch.float64, device="cuda") * (m * n / nnz)
    for c0 in range(0, nnz, 1 << 23):
        c1 = min(nnz, c0 + (1 << 23))
        vals[c0:c1] += (u[rows[c0:c1]] * v[cols[c0:c1].long()] * sig).sum(1)
    del rows, u, v
    return indptr, cols, vals


def dense_columns(m, n, nd, seed, dens=(0.1, 0.4), rest=0.004):
    """nd columns of densities uniform in `dens`, the others of density `rest`;
    values log1p(Poisson(3) + 1): a matrix with a dense-column split."""
    rng = np.random.default_rng(seed)
    dcols = rng.choice(n, nd, replace=False)
    p = np.full(n, rest)
    p[dcols] = rng.uniform(dens[0], dens[1], nd)
    mask = rng.random((m, n)) < p[None, :]
    r, c = np.nonzero(mask)
    v = np.log1p(rng.poisson(3.0, len(r)) + 1.0)
    return from_scipy(sp.csr_matrix((v, (r, c)), shape=(m, n)))
