"""SMat operator entry points on the GPU against the checker: svd_opa / svd_opb
(src/lanczos/mod.rs:311-319, 1427-1700) for CSR, CSC, COO and masked views,
and the dense products multiply_with_dense / multiply_transposed_by_dense
(src/lanczos/masked.rs:265-733).  Tolerance 1e-13 relative to the largest
entry (FMA and summation order differ)."""
import numpy as np
import pytest

import matrices as M
import oracle as O
from gpu_util import oracle_args, upload

pytestmark = pytest.mark.gpu


def close(a, b, tol=1e-13):
    scale = max(np.max(np.abs(b)), 1e-300)
    np.testing.assert_allclose(a, b, rtol=0, atol=tol * scale)


@pytest.mark.parametrize("kind", ["csr", "csc", "coo", "masked"])
@pytest.mark.parametrize("shape", [(50, 30), (300, 700), (1000, 64)])
def test_opa_opb(kind, shape):
    A = M.uniform(shape[0], shape[1], 0.05, 7)
    mask = (np.random.default_rng(2).random(shape[1]) < 0.7).astype(np.uint8) if kind == "masked" else None
    h = upload(kind, A, mask)
    ncols = int(mask.sum()) if mask is not None else shape[1]
    rng = np.random.default_rng(3)
    x = rng.standard_normal(ncols)
    y = rng.standard_normal(shape[0])
    ka = "masked" if kind == "masked" else kind
    OA = oracle_args(kind, A)
    close(h.svd_opa(x), O.opa(ka, OA, x, False, mask=mask))
    close(h.svd_opa(y, transposed=True), O.opa(ka, OA, y, True, mask=mask))
    close(h.svd_opb(x), O.opa(ka, OA, O.opa(ka, OA, x, False, mask=mask), True, mask=mask))


def test_power_law_rows():
    # rows from 1 to 3000 entries exercise every group width of the row gather
    rng = np.random.default_rng(11)
    m, n = 4000, 5000
    k = np.minimum((rng.pareto(1.2, m) * 5 + 1).astype(int), 3000)
    import scipy.sparse as sp
    rows = np.repeat(np.arange(m), k)
    cols = np.concatenate([rng.choice(n, kk, replace=False) for kk in k])
    S = sp.csr_matrix((rng.standard_normal(len(rows)), (rows, cols)), shape=(m, n))
    A = M.from_scipy(S)
    h = upload("csr", A)
    x = rng.standard_normal(n)
    close(h.svd_opa(x), S @ x, 1e-12)
    y = rng.standard_normal(m)
    close(h.svd_opa(y, transposed=True), S.T @ y, 1e-12)


@pytest.mark.parametrize("l", [1, 7, 32, 60, 150])
def test_dense_products(l):
    A = M.uniform(400, 250, 0.04, 21)
    mask = (np.random.default_rng(4).random(250) < 0.5).astype(np.uint8)
    rng = np.random.default_rng(5)
    for h, mk in [(upload("csr", A), np.ones(250, np.uint8)), (upload("masked", A, mask), mask)]:
        nm = int(mk.sum())
        X = rng.standard_normal((nm, l))
        Y = rng.standard_normal((400, l))
        close(h.multiply_with_dense(X), O.masked_dense(A, mk, "AX", X), 1e-12)
        close(h.multiply_with_dense(Y, transpose_self=True), O.masked_dense(A, mk, "ATX", Y), 1e-12)
        close(h.multiply_transposed_by_dense(Y), O.masked_dense(A, mk, "XTA", Y), 1e-12)


@pytest.mark.parametrize("l", [3, 130, 300])
def test_centred_products_and_column_means(l):
    """compute_column_means (masked.rs:240-263) and the centred products of
    src/utils.rs:29-32 as exact products of A - 1 means^T, against numpy;
    l above 128 crosses the 128-column slices of the rank-1 correction."""
    A = M.uniform(400, 180, 0.1, 17)
    mk = (np.random.default_rng(5).random(180) < 0.6).astype(np.uint8)
    nm = int(mk.sum())
    D = M.to_scipy(A).toarray()[:, mk.astype(bool)]
    h = upload("masked", A, mk)
    mu = h.column_means()
    close(mu, D.mean(0))
    rng = np.random.default_rng(9)
    means = mu + rng.standard_normal(nm)  # any means vector, not only the column means
    Dc = D - means[None, :]
    X = rng.standard_normal((nm, l))
    Y = rng.standard_normal((400, l))
    close(h.multiply_with_dense_centered(X, means), Dc @ X, 1e-12)
    close(h.multiply_with_dense_centered(Y, means, transpose_self=True), Dc.T @ Y, 1e-12)
    close(h.multiply_transposed_by_dense_centered(Y, means), Y.T @ Dc, 1e-12)
    with pytest.raises(Exception):
        h.multiply_with_dense_centered(X, means[:-1])


def test_empty_rows_and_columns():
    import scipy.sparse as sp
    S = sp.csr_matrix(([1.0, 2.0, 3.0], ([0, 5, 5], [3, 3, 9])), shape=(8, 12))
    A = M.from_scipy(S)
    h = upload("csr", A)
    x = np.arange(12.0)
    close(h.svd_opa(x), S @ x)
    close(h.svd_opa(np.ones(8), transposed=True), S.T @ np.ones(8))


@pytest.mark.parametrize("l", [1, 8, 30, 40, 60, 64, 96])
@pytest.mark.parametrize("transpose", [False, True])
@pytest.mark.parametrize("impl", ["lean", "seg", "tma"])
def test_device_fp32_spmm_against_numpy(l, transpose, impl, monkeypatch):
    """svdb_multiply_with_dense_device with FP32 operands against numpy on
    FP32-rounded inputs, through the default kernels (k_spmm_f32 where l is a
    multiple of 4 up to 64, else k_spmm_seg), the register-gather kernel
    (SVDB_SPMM=seg) and the opt-in tensor-memory gather kernel (SVDB_SPMM=tma;
    it takes rows that are 16-byte multiples of at most 64 columns); includes a
    row long enough to be split into several segments."""
    import torch
    if impl == "lean":
        monkeypatch.delenv("SVDB_SPMM", raising=False)
    else:
        monkeypatch.setenv("SVDB_SPMM", impl)
    from single_svdlib import _abi
    from single_svdlib._core import check
    rng = np.random.default_rng(l)
    D = (rng.random((700, 5000)) < 0.01) * rng.standard_normal((700, 5000))
    D[3, :] = rng.standard_normal(5000)        # 5000 entries: three segments of the plan
    D[:, 7] = rng.standard_normal(700)         # a dense column for A^T
    A = M.dense(D)
    h = upload("csr", A)
    rows_in = 700 if transpose else 5000
    X = rng.standard_normal((rows_in, l)).astype(np.float32)
    Df = D.astype(np.float32).astype(np.float64)
    ref = (Df.T if transpose else Df) @ X.astype(np.float64)
    tx = torch.from_numpy(X).cuda()
    ty = torch.empty((5000 if transpose else 700, l), dtype=torch.float32, device="cuda")
    check(_abi.lib().svdb_multiply_with_dense_device(h.handle, tx.data_ptr(), l, ty.data_ptr(), int(transpose), 1,
                                                     None))
    torch.cuda.synchronize()
    got = ty.cpu().numpy().astype(np.float64)
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() <= 2e-6 * scale


@pytest.mark.parametrize("rows", [5, 31, 1000, 10007, 200000])
@pytest.mark.parametrize("c", [1, 8, 33, 60, 64])
def test_gram_device(rows, c):
    """svdb_gram_device: X^T X on the tensor cores (SVDB_MIXED: 3xTF32 products,
    FP32 accumulation over at most 256 rows per block, FP64 across blocks)
    within 1e-5 of the largest entry (256 FP32 additions: 256 * 2^-24 = 1.5e-5
    at most), and in FP64 on the CUDA cores within 1e-12, against numpy."""
    import torch
    from single_svdlib import _abi
    from single_svdlib._core import check
    rng = np.random.default_rng(rows + c)
    X = rng.standard_normal((rows, c)) * np.exp(rng.standard_normal(c))  # columns of different scales
    ref = X.T @ X
    tx = torch.from_numpy(X).cuda()
    for prec, tol in ((1, 1e-5), (0, 1e-12)):
        tg = torch.empty((c, c), dtype=torch.float64, device="cuda")
        check(_abi.lib().svdb_gram_device(tx.data_ptr(), rows, c, tg.data_ptr(), prec, None))
        got = tg.cpu().numpy()
        assert np.abs(got - ref).max() <= tol * np.abs(ref).max(), (prec, np.abs(got - ref).max())


def test_gram_device_empty_and_limits():
    import torch
    from single_svdlib import UnsupportedError, _abi
    from single_svdlib._core import check
    tx = torch.zeros((0, 4), dtype=torch.float64, device="cuda")
    tg = torch.full((4, 4), 7.0, dtype=torch.float64, device="cuda")
    check(_abi.lib().svdb_gram_device(tx.data_ptr() or 1, 0, 4, tg.data_ptr(), 1, None))
    assert not tg.cpu().numpy().any()
    big = torch.zeros((10, 65), dtype=torch.float64, device="cuda")
    with pytest.raises(UnsupportedError):
        check(_abi.lib().svdb_gram_device(big.data_ptr(), 10, 65, tg.data_ptr(), 1, None))
