"""Batches of masked column subsets (svdb_batch_*): each subset's result
against randomized_svd on MaskedCSRMatrix::with_columns with the same seed
(f64: singular values 1e-10 relative, leading singular subspaces to 1e-8;
FP32 products: 1e-6 against the f64 batch), the with_columns semantics
(order and duplicates ignored, bounds), the captured graph against direct
launches, and the autotuner's reported choice."""
import numpy as np
import pytest

import matrices as M
from gpu_util import subspace_cos, upload
from single_svdlib import MaskedCSRMatrix, ShapeError, UnsupportedError, _abi, randomized
from single_svdlib.randomized import PowerIterationNormalizer as PIN
from single_svdlib.randomized import RandomizedBatch

pytestmark = pytest.mark.gpu


def subsets_of(n, count, lo, hi, seed):
    rng = np.random.default_rng(seed)
    return [rng.choice(n, rng.integers(lo, hi + 1), replace=False) for _ in range(count)]


def single(A, h, cols, rank, over, q, norm, seed, precision):
    mv = MaskedCSRMatrix.with_columns(h, cols)
    return randomized.randomized_svd(mv, rank, over, q, norm, False, seed, False, precision=precision)


@pytest.mark.parametrize("norm", [PIN.QR, PIN.LU, PIN.None_])
@pytest.mark.parametrize("q", [0, 2])
def test_batch_f64_matches_single_calls(norm, q):
    A = M.lowrank_plus_noise(500, 300, 10, 1e-2, 12, density=0.3)
    h = upload("csr", A)
    subs = subsets_of(300, 7, 40, 200, 3)
    rank, over, seed = 6, 4, 11
    got = randomized.randomized_svd_batch(h, subs, rank, over, q, norm, seed, precision="f64")
    assert len(got) == len(subs)
    tol = 1e-10 if norm == PIN.QR else 1e-8
    for cols, g in zip(subs, got):
        ref = single(A, h, cols, rank, over, q, norm, seed, "f64")
        assert g.u.shape == ref.u.shape == (500, rank)
        assert g.vt.shape == ref.vt.shape == (rank, len(np.unique(cols)))
        np.testing.assert_allclose(g.s, ref.s, rtol=tol)
        k = 3
        assert np.all(subspace_cos(g.u[:, :k], ref.u[:, :k]) > 1 - 1e-8)
        assert np.all(subspace_cos(g.vt[:k].T, ref.vt[:k].T) > 1 - 1e-8)


def test_batch_mixed_against_f64_and_graph_against_direct():
    A = M.lowrank_plus_noise(800, 400, 12, 1e-2, 5, density=0.2)
    h = upload("csr", A)
    subs = subsets_of(400, 12, 60, 300, 9)
    f64 = randomized.randomized_svd_batch(h, subs, 8, 6, 2, PIN.QR, 3, precision="f64")
    b1 = RandomizedBatch(h, subs, 8, 6, 2, PIN.QR, 3, precision="mixed", use_graph=True)
    b2 = RandomizedBatch(h, subs, 8, 6, 2, PIN.QR, 3, precision="mixed", use_graph=False)
    g1, g2 = b1.run(), b2.run()
    for a, b, c in zip(g1, g2, f64):
        np.testing.assert_array_equal(a.s, b.s)          # same kernels, same order
        np.testing.assert_array_equal(a.u, b.u)
        np.testing.assert_allclose(a.s, c.s, rtol=1e-6)  # FP32 products vs f64
    info = b1.info()
    assert info["count"] == len(subs)
    assert info["subsets_per_row_item"] in (1, 2, 4, 8)
    assert info["graph_nodes"] > 0 and info["kernels_per_run"] > 0
    l0 = _abi.lib().svdb_kernel_launches()
    b1.run()
    assert _abi.lib().svdb_kernel_launches() - l0 == info["kernels_per_run"]
    # a second run replays the same graph: identical results
    g3 = b1.run()
    for a, b in zip(g1, g3):
        np.testing.assert_array_equal(a.s, b.s)
    b1.close()
    b2.close()


def test_batch_with_columns_semantics():
    A = M.uniform(300, 120, 0.2, 8, -1.0, 1.0)
    h = upload("csr", A)
    base = np.arange(10, 90, 2)
    messy = np.concatenate([base[::-1], base[:5]])     # unsorted, with duplicates
    got = randomized.randomized_svd_batch(h, [base, messy], 5, 5, 1, PIN.QR, 2, precision="f64")
    np.testing.assert_array_equal(got[0].s, got[1].s)
    np.testing.assert_array_equal(got[0].vt, got[1].vt)
    with pytest.raises(ShapeError):
        randomized.randomized_svd_batch(h, [np.array([0, 120] + list(range(1, 20)))], 5, 5, 1, seed=2)
    with pytest.raises(UnsupportedError):  # fewer columns than rank + oversamples
        randomized.randomized_svd_batch(h, [np.arange(8)], 5, 5, 1, seed=2)
    with pytest.raises(UnsupportedError):  # a masked view is not a batch parent
        randomized.randomized_svd_batch(MaskedCSRMatrix.with_columns(h, base), [base[:20]], 5, 5, 1, seed=2)


def test_batch_uneven_subsets_and_csc_parent():
    A = M.poisson_rows(1200, 500, 30, 21)
    h = upload("csc", A)
    subs = subsets_of(500, 20, 30, 480, 4)   # sizes from 30 to 480 columns
    got = randomized.randomized_svd_batch(h, subs, 10, 10, 1, PIN.QR, 5, precision="f64")
    for cols, g in zip(subs[:5], got[:5]):
        ref = single(A, upload("csr", A), cols, 10, 10, 1, PIN.QR, 5, "f64")
        np.testing.assert_allclose(g.s, ref.s, rtol=1e-10)


def test_batch_dense_split_against_gather_and_f64(monkeypatch):
    """Under SVDB_MIXED the dense columns of every subset go through one GEMM
    over all subsets (the dense-column split); the rest through the batch's
    gathers.  Against the same batch with the split off and single FP64 calls."""
    import ctypes as C
    A = M.dense_columns(5000, 2400, 300, 17)
    subs = subsets_of(2400, 9, 150, 2000, 6)
    rank, over, q, seed = 12, 8, 2, 4
    monkeypatch.setenv("SVDB_DENSE_SPLIT", "1")  # the split is opt-in
    h = upload("csr", A)
    got = randomized.randomized_svd_batch(h, subs, rank, over, q, PIN.QR, seed, precision="mixed")
    nd, nnz = C.c_uint64(0), C.c_uint64(0)
    assert _abi.lib().svdb_dense_split_info(h.handle, C.byref(nd), C.byref(nnz)) == 0
    assert nd.value == 300 and nnz.value > 0
    monkeypatch.setenv("SVDB_DENSE_SPLIT", "0")
    h2 = upload("csr", A)
    gat = randomized.randomized_svd_batch(h2, subs, rank, over, q, PIN.QR, seed, precision="mixed")
    assert _abi.lib().svdb_dense_split_info(h2.handle, C.byref(nd), C.byref(nnz)) == 0 and nd.value == 0
    for cols, g, r in list(zip(subs, got, gat))[:4]:
        ref = single(A, h2, cols, rank, over, q, PIN.QR, seed, "f64")
        assert np.max(np.abs(g.s - ref.s) / ref.s) < 1e-6
        assert np.max(np.abs(r.s - ref.s) / ref.s) < 1e-6
