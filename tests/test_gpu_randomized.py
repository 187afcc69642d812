"""randomized_svd on the GPU against the checker with the same Omega
(src/randomized/mod.rs:24-199).  QR is CholeskyQR2 here and Householder in the
checker, so column signs may differ: singular values are compared directly
(1e-10 relative, f64), singular vectors through principal angles (cosines
within 1e-8 of 1 for the leading, well-separated ones)."""
import numpy as np
import pytest

import matrices as M
import oracle as O
from gpu_util import subspace_cos, upload
from single_svdlib import MaskedCSRMatrix, randomized
from single_svdlib.randomized import PowerIterationNormalizer as PIN

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("norm", ["QR", "LU", "None"])
@pytest.mark.parametrize("q", [0, 1, 3])
def test_parity_with_checker(norm, q):
    A = M.lowrank_plus_noise(400, 150, 12, 1e-2, 31, density=0.3)
    l = 10 + 6
    om = M.omega(150, l, 5)
    ref = O.randomized(A, 10, 6, q, norm, omega=om)
    got = randomized.randomized_svd(upload("csr", A), 10, 6, q, getattr(PIN, norm if norm != "None" else "None_"),
                                    False, 7, False, omega=om)
    assert got.d == ref["d"] == 10
    assert got.u.shape == (400, 10) and got.vt.shape == (10, 150)
    tol = 1e-10 if norm == "QR" else 1e-7
    np.testing.assert_allclose(got.s, ref["s"], rtol=tol)
    k = 5
    assert np.all(subspace_cos(got.u[:, :k], ref["u"][:, :k]) > 1 - 1e-8)
    assert np.all(subspace_cos(got.vt[:k].T, ref["vt"][:k].T) > 1 - 1e-8)


def test_all_true_masked_and_diagnostics():
    A = M.uniform(300, 90, 0.1, 41)
    om = M.omega(90, 15, 1)
    mv = MaskedCSRMatrix(upload("csr", A), np.ones(90, np.uint8))
    got = randomized.randomized_svd(mv, 10, 5, 2, PIN.QR, False, 42, False, omega=om)
    ref = O.randomized(A, 10, 5, 2, "QR", omega=om)
    np.testing.assert_allclose(got.s, ref["s"], rtol=1e-10)
    dg = got.diagnostics
    assert (dg.non_zero, dg.dimensions, dg.iterations, dg.lanczos_steps, dg.random_seed) == (len(A["data"]), 10, 2,
                                                                                              0, 42)
    assert dg.significant_values == dg.singular_values == dg.ritz_values_stabilized == 10
    # descending, positive (randomized/mod.rs:683-689)
    assert np.all(np.diff(got.s) <= 0) and np.all(got.s > 0)
    # recompose works on the m x d orientation
    assert got.recompose().shape == (300, 90)


def test_real_mask():
    A = M.uniform(250, 120, 0.1, 43)
    mask = (np.random.default_rng(2).random(120) < 0.5).astype(np.uint8)
    nm = int(mask.sum())
    om = M.omega(nm, 12, 3)
    mv = MaskedCSRMatrix(upload("csr", A), mask)
    got = randomized.randomized_svd(mv, 8, 4, 2, PIN.QR, False, 1, False, omega=om)
    ref = O.randomized(A, 8, 4, 2, "QR", omega=om, mask=mask)
    np.testing.assert_allclose(got.s, ref["s"], rtol=1e-10)


def test_mixed_precision_error_is_stated():
    A = M.lowrank_plus_noise(500, 200, 15, 1e-2, 51, density=0.2)
    om = M.omega(200, 25, 2)
    f64 = randomized.randomized_svd(upload("csr", A), 15, 10, 3, PIN.QR, False, 1, False, omega=om)
    mix = randomized.randomized_svd(upload("csr", A), 15, 10, 3, PIN.QR, False, 1, False, omega=om,
                                    precision="mixed")
    rel = np.max(np.abs(mix.s - f64.s) / f64.s)
    assert rel < 1e-6, rel


@pytest.mark.parametrize("fmt", ["csr", "masked"])
def test_mixed_panel_spmm_matches_segment_spmm(fmt, monkeypatch):
    """The FP32 products through the panel kernel (X staged in shared memory by
    panels of 384 rows) against the segment kernel, on a matrix with rows and
    columns long enough to be left to the segment kernel (more than 2048
    entries) and an empty row."""
    rng = np.random.default_rng(77)
    m, n = 6000, 2600
    lens = np.minimum(n, rng.lognormal(np.log(50), 0.7, m).astype(int))
    lens[3], lens[9], lens[10] = n, 0, 2500
    rows = np.repeat(np.arange(m), lens)
    cols = np.concatenate([rng.choice(n, k, replace=False) for k in lens])
    dense_col = np.arange(0, m, 2)  # column 7: 3000 entries
    rows = np.concatenate([rows, dense_col])
    cols = np.concatenate([cols, np.full(len(dense_col), 7)])
    import scipy.sparse as sp
    S = sp.csr_matrix((rng.random(len(rows)) + 0.5, (rows, cols)), shape=(m, n))
    S.sum_duplicates()
    S.sort_indices()
    A = M.from_scipy(S)
    mask = (np.arange(n) % 5 != 2).astype(np.uint8) if fmt == "masked" else None
    nc = int(mask.sum()) if mask is not None else n
    om = M.omega(nc, 16, 4)
    mat = lambda: MaskedCSRMatrix(upload("csr", A), mask) if mask is not None else upload("csr", A)  # noqa: E731
    res = {}
    for impl in ("seg", "panel"):
        monkeypatch.setenv("SVDB_SPMM", impl)
        res[impl] = randomized.randomized_svd(mat(), 10, 6, 2, PIN.QR, False, 1, False, omega=om,
                                              precision="mixed")
    f64 = randomized.randomized_svd(mat(), 10, 6, 2, PIN.QR, False, 1, False, omega=om)
    assert np.max(np.abs(res["panel"].s - res["seg"].s) / res["seg"].s) < 2e-6
    assert np.max(np.abs(res["panel"].s - f64.s) / f64.s) < 1e-6
    assert np.all(subspace_cos(res["panel"].u[:, :5], f64.u[:, :5]) > 1 - 1e-6)

    # the plan built through a view belongs to the parent: the view may go first
    monkeypatch.setenv("SVDB_SPMM", "panel")
    parent = upload("csr", A)
    view = MaskedCSRMatrix(parent, np.ones(n, np.uint8))
    r = randomized.randomized_svd(view, 10, 6, 2, PIN.QR, False, 1, False, omega=M.omega(n, 16, 4),
                                  precision="mixed")
    assert np.all(np.isfinite(r.s))
    view.close()
    parent.close()


def test_device_omega_is_seeded():
    A = M.uniform(200, 80, 0.1, 44)
    r1 = randomized.randomized_svd(upload("csr", A), 5, 5, 1, PIN.QR, False, 9, False)
    r2 = randomized.randomized_svd(upload("csr", A), 5, 5, 1, PIN.QR, False, 9, False)
    np.testing.assert_array_equal(r1.s, r2.s)
    truth = np.linalg.svd(M.to_scipy(A).toarray(), compute_uv=False)[:5]
    assert np.max(np.abs(r1.s - truth) / truth) < 0.3


@pytest.mark.parametrize("seed", [0, 7, 2**40 + 3])
def test_device_omega_is_the_restated_stream(seed):
    # the seeded Omega drawn on the device is the stream oracle.omega_stream restates
    A = M.lowrank_plus_noise(400, 150, 12, 1e-2, 33, density=0.3)
    got = randomized.randomized_svd(upload("csr", A), 10, 6, 2, PIN.QR, False, seed, False)
    ref = O.randomized(A, 10, 6, 2, "QR", omega=O.omega_stream(seed, 150, 16))
    np.testing.assert_allclose(got.s, ref["s"], rtol=1e-10)


def test_small_wide_and_rank_edge_cases():
    # l larger than ncols: Q has min(rows, l) columns (nalgebra's thin QR)
    A = M.uniform(30, 8, 0.6, 45)
    got = randomized.randomized_svd(upload("csr", A), 5, 10, 2, PIN.QR, False, 3, False)
    truth = np.linalg.svd(M.to_scipy(A).toarray(), compute_uv=False)[:5]
    np.testing.assert_allclose(got.s, truth, rtol=1e-8)


@pytest.mark.parametrize("fmt", ["csr", "csc", "masked"])
@pytest.mark.parametrize("norm", ["QR", "LU"])
def test_mean_center_parity_with_checker(fmt, norm):
    # A - 1 mu^T through the rank-1 corrected products, same Omega as the checker
    A = M.uniform(350, 140, 0.15, 61, low=0.0, high=4.0)
    mask = (np.random.default_rng(8).random(140) < 0.7).astype(np.uint8) if fmt == "masked" else None
    nc = int(mask.sum()) if mask is not None else 140
    om = M.omega(nc, 16, 6)
    mat = MaskedCSRMatrix(upload("csr", A), mask) if mask is not None else upload(fmt, A)
    got = randomized.randomized_svd(mat, 10, 6, 2, getattr(PIN, norm), True, 3, False, omega=om)
    ref = O.randomized(A, 10, 6, 2, norm, omega=om, mask=mask, mean_center=True)
    np.testing.assert_allclose(got.s, ref["s"], rtol=1e-10 if norm == "QR" else 1e-7)
    assert np.all(subspace_cos(got.u[:, :4], ref["u"][:, :4]) > 1 - 1e-8)
    assert np.all(subspace_cos(got.vt[:4].T, ref["vt"][:4].T) > 1 - 1e-8)
    # U spans columns of the centred matrix: every column of U sums to zero
    assert np.max(np.abs(got.u.sum(0))) < 1e-10 * np.sqrt(350)


def test_mean_center_matches_dense_centred_svd():
    # sketch as wide as the matrix: the exact SVD of A - 1 mu^T, in both precisions
    A = M.lowrank_plus_noise(600, 90, 6, 1e-2, 62, density=0.4)
    Ad = M.to_scipy(A).toarray() + 0.0
    U, s, Vt = np.linalg.svd(Ad - Ad.mean(0), full_matrices=False)
    got = randomized.randomized_svd(upload("csr", A), 6, 84, 1, PIN.QR, True, 5, False)
    np.testing.assert_allclose(got.s, s[:6], rtol=1e-10)
    assert np.all(subspace_cos(got.vt.T, Vt[:6].T) > 1 - 1e-10)
    mix = randomized.randomized_svd(upload("csr", A), 6, 84, 1, PIN.QR, True, 5, False, precision="mixed")
    assert np.max(np.abs(mix.s - s[:6]) / s[:6]) < 1e-6


def test_mean_center_constant_columns():
    # a constant column has zero variance: centring removes it exactly
    Z = M.dense(np.tile(np.arange(1.0, 6.0), (40, 1)))
    got = randomized.randomized_svd(upload("csr", Z), 3, 2, 1, PIN.QR, True, 3, False)
    assert np.all(np.abs(got.s) < 1e-12 * np.sqrt(40 * 55.0))  # relative to ||Z||_F


def test_rank_deficient_input_takes_the_shifted_qr():
    # rank 5 < l = 15: the Gram of Y is singular, so CholeskyQR needs its shift;
    # the leading singular values must still be exact and the rest ~0
    rng = np.random.default_rng(71)
    Mx = (rng.standard_normal((200, 5)) * np.geomspace(10, 1, 5)) @ rng.standard_normal((5, 80))
    A = M.dense(Mx)
    got = randomized.randomized_svd(upload("csr", A), 10, 5, 2, PIN.QR, False, 5, False)
    truth = np.linalg.svd(Mx, compute_uv=False)
    np.testing.assert_allclose(got.s[:5], truth[:5], rtol=1e-9)
    assert np.all(np.abs(got.s[5:]) < 1e-8 * truth[0])
    assert np.all(np.isfinite(got.u)) and np.all(np.isfinite(got.vt))
