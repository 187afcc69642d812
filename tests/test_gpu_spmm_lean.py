"""The lean gather kernels (k_spmm_f32, k_spmm_lean<double>, csrc/spmm.cu;
k_b_rows_lean, k_b_cols_lean, csrc/batch.cu) against the kernels they replace.

- Single products at l = 60: the lean kernels keep k_spmm_seg's lane groups
  and summation order, so A X and A^T Y must be bit-identical to
  SVDB_SPMM=seg, FP32 and FP64, on a matrix with rows split into several
  segments of the plan (above 2,048 entries) and empty rows.
- Batch products: SVDB_MIXED batches at l = 32 (quarter-warp lane groups) and
  l = 64 (half-warp groups) through the lean kernels against the same batch
  through the warp-per-entry kernels (SVDB_BATCH_SPMM=warp) and against an
  FP64 batch, sigma within 1e-6.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import matrices as M
from gpu_util import upload
from single_svdlib import _abi, randomized
from single_svdlib._core import check
from single_svdlib.randomized import PowerIterationNormalizer as PIN

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def long_rows():
    rng = np.random.default_rng(31)
    m, n = 3000, 8000
    lens = np.minimum((rng.pareto(1.1, m) * 20 + 1).astype(int), n)
    lens[:3] = [7000, 4500, 0]
    lens[50:60] = 0
    rows = np.repeat(np.arange(m), lens)
    cols = np.concatenate([rng.choice(n, k, replace=False) for k in lens])
    S = sp.csr_matrix((rng.standard_normal(len(rows)), (rows, cols)), shape=(m, n))
    S.sort_indices()
    return M.from_scipy(S)


def products(h, A, l, dtype, precision):
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    X = torch.randn(A["ncols"], l, dtype=dtype, device="cuda", generator=g)
    Yi = torch.randn(A["nrows"], l, dtype=dtype, device="cuda", generator=g)
    Y = torch.full((A["nrows"], l), float("nan"), dtype=dtype, device="cuda")
    Z = torch.full((A["ncols"], l), float("nan"), dtype=dtype, device="cuda")
    L = _abi.lib()
    check(L.svdb_multiply_with_dense_device(h.handle, X.data_ptr(), l, Y.data_ptr(), 0, precision, None))
    check(L.svdb_multiply_with_dense_device(h.handle, Yi.data_ptr(), l, Z.data_ptr(), 1, precision, None))
    torch.cuda.synchronize()
    return Y.cpu().numpy(), Z.cpu().numpy()


@pytest.mark.parametrize("precision", [0, 1])
def test_bit_identical_to_segment_kernel(long_rows, precision, monkeypatch):
    import torch
    dtype = torch.float32 if precision == 1 else torch.float64
    monkeypatch.delenv("SVDB_SPMM", raising=False)
    lean = products(upload("csr", long_rows), long_rows, 60, dtype, precision)
    monkeypatch.setenv("SVDB_SPMM", "seg")
    seg = products(upload("csr", long_rows), long_rows, 60, dtype, precision)
    for a, b in zip(lean, seg):
        assert np.all(np.isfinite(a))
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("rank,over", [(20, 12), (40, 24)])
def test_lean_batch_against_warp_kernels_and_f64(rank, over, monkeypatch):
    A = M.lowrank_plus_noise(3000, 1200, 30, 1e-2, 8, density=0.15)
    rng = np.random.default_rng(2)
    subs = [np.sort(rng.choice(1200, k, replace=False)) for k in (100, 450, 1199, 700, 260)]
    q, seed = 2, 9
    h = upload("csr", A)
    monkeypatch.delenv("SVDB_BATCH_SPMM", raising=False)
    lean = randomized.randomized_svd_batch(h, subs, rank, over, q, PIN.QR, seed, precision="mixed")
    monkeypatch.setenv("SVDB_BATCH_SPMM", "warp")
    warp = randomized.randomized_svd_batch(h, subs, rank, over, q, PIN.QR, seed, precision="mixed")
    f64 = randomized.randomized_svd_batch(h, subs, rank, over, q, PIN.QR, seed, precision="f64")
    for a, b, c in zip(lean, warp, f64):
        assert np.max(np.abs(a.s - c.s) / c.s) < 1e-6
        assert np.max(np.abs(a.s - b.s) / b.s) < 1e-6
