"""Parity at the workloads' own sizes, against the checker (oracle/).

- The randomized_svd workload (100,000 x 30,000 count-like CSR, 65 M nnz,
  rank 50 + 10, 3 power iterations, QR, seed 7; src/randomized/mod.rs:24-199):
  the CUDA solve draws Omega on the device from the seed, the checker gets the
  same stream restated on the host.  FP64 sigma within 1e-10, FP32 products
  (SVDB_MIXED) within 1e-6, the bound the mixed form is held to.
- The large LAS2 workload (1,000,000 x 200,000, ~200 M nnz): a step-capped run
  (iterations 60, dimensions 10, SVDLIBC semantics; src/legacy.rs:569-654),
  alpha/beta of every step within 1e-10 and sigma of the capped run within
  1e-10 (FP64); the FP32-value form within 1e-6.
- The batch workload (column subsets of the count-like matrix, rank 30 + 10,
  2 power iterations; MaskedCSRMatrix::with_columns, src/lanczos/masked.rs:48-66):
  four of the 256 subsets against the checker's randomized_svd on the same
  masked view and the same Omega stream.

These take minutes (the checker solves the full matrices on the host cores).
"""
import numpy as np
import pytest

import matrices as M
import oracle as O
from gpu_util import subspace_cos
from single_svdlib import CsrMatrix, MaskedCSRMatrix, randomized
from single_svdlib.lanczos import las2_traced
from single_svdlib.randomized import PowerIterationNormalizer as PIN
from single_svdlib.randomized import RandomizedBatch

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


@pytest.fixture(scope="module")
def count_like():
    indptr, cols, vals = M.count_like(100_000, 30_000, 2024)
    return {"nrows": 100_000, "ncols": 30_000, "indptr": indptr, "indices": cols, "data": vals}


@pytest.fixture(scope="module", autouse=True)
def _threads():
    import os
    O.set_threads(len(os.sched_getaffinity(0)))


def test_randomized_workload_against_checker(count_like):
    A = count_like
    rank, over, q, seed = 50, 10, 3, 7
    ref = O.randomized(A, rank, over, q, "QR", omega=O.omega_stream(seed, A["ncols"], rank + over))
    parent = CsrMatrix(A["nrows"], A["ncols"], A["indptr"], A["indices"], A["data"])
    view = MaskedCSRMatrix(parent, np.ones(A["ncols"], np.uint8))
    got = {p: randomized.randomized_svd(view, rank, over, q, PIN.QR, False, seed, False, precision=p)
           for p in ("f64", "mixed")}
    err = {p: float(np.max(np.abs(g.s - ref["s"]) / ref["s"])) for p, g in got.items()}
    print("sigma rel err vs checker:", err)
    assert err["f64"] < 1e-10, err
    assert err["mixed"] < 1e-6, err
    # leading singular vectors: the gap after sigma_10 is wide on this matrix
    k = 10
    for p, tol in (("f64", 1e-8), ("mixed", 1e-6)):
        assert np.all(subspace_cos(got[p].u[:, :k], ref["u"][:, :k]) > 1 - tol), p
        assert np.all(subspace_cos(got[p].vt[:k].T, ref["vt"][:k].T) > 1 - tol), p


def test_batch_subsets_against_checker(count_like):
    A = count_like
    n = A["ncols"]
    rng = np.random.default_rng(11)
    sizes = rng.integers(500, 20001, 256)
    subs = [np.sort(rng.choice(n, int(k), replace=False)) for k in sizes]
    pick = [0, 85, 170, 255]
    rank, over, q, seed = 30, 10, 2, 7
    parent = CsrMatrix(A["nrows"], n, A["indptr"], A["indices"], A["data"])
    mixed = RandomizedBatch(parent, subs, rank, over, q, PIN.QR, seed, precision="mixed").run()
    f64 = RandomizedBatch(parent, [subs[i] for i in pick], rank, over, q, PIN.QR, seed, precision="f64").run()
    for j, b in enumerate(pick):
        mask = np.zeros(n, np.uint8)
        mask[subs[b]] = 1
        ref = O.randomized(A, rank, over, q, "QR", omega=O.omega_stream(seed, len(subs[b]), rank + over), mask=mask)
        e64 = float(np.max(np.abs(f64[j].s - ref["s"]) / ref["s"]))
        emx = float(np.max(np.abs(mixed[b].s - ref["s"]) / ref["s"]))
        print(f"subset {b} ({len(subs[b])} columns): sigma rel err f64 {e64:.2e}, mixed {emx:.2e}")
        assert e64 < 1e-10, (b, e64)
        assert emx < 1e-6, (b, emx)


def test_large_las2_capped_against_checker():
    torch = pytest.importorskip("torch")
    ip, ix, v = M.zipf_planted_device(torch, 1_000_000, 200_000, 3)
    A = {"nrows": 1_000_000, "ncols": 200_000, "indptr": ip.cpu().numpy(),
         "indices": ix.cpu().numpy().astype(np.int64), "data": v.cpu().numpy()}
    del ip, ix, v
    torch.cuda.empty_cache()
    dims, iters, seed = 10, 60, 42
    ref = O.las2("csr", A, dims, iters, seed=seed, legacy=True)
    mat = CsrMatrix(A["nrows"], A["ncols"], A["indptr"], A["indices"], A["data"])
    for prec, tol in (("f64", 1e-10), ("mixed", 1e-6)):
        got = las2_traced(mat, dims, iters, random_seed=seed, algorithm="legacy", precision=prec)
        assert got["error"] is None, got["error"]
        assert got["steps"] == ref["steps"]
        k = ref["steps"] + 1
        scale = np.max(np.abs(ref["alf"][:k]))
        da = np.max(np.abs(got["alf"][:k] - ref["alf"][:k])) / scale
        db = np.max(np.abs(got["bet"][:k] - ref["bet"][:k])) / scale
        rec = got["rec"]
        assert rec.d == ref["d"]
        ds = float(np.max(np.abs(rec.s - ref["s"]) / np.max(ref["s"]))) if rec.d else 0.0
        print(f"{prec}: steps {got['steps']}, alpha {da:.2e}, beta {db:.2e}, sigma {ds:.2e}")
        assert da < tol and db < tol and ds < tol, (prec, da, db, ds)
    mat.close()
