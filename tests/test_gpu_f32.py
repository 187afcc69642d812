"""The crate's solvers at T = f32 (impl SvdFloat for f32, src/utils.rs:87-99)
on the GPU, against the checker built for T = f32 (oracle/liboracle_f32.so).

The GPU keeps FP64 sums and recurrences at T = f32; what it takes from f32
is what decides the run: f32 epsilon in every tolerance, kappa clamped to f32
eps34, the start vector and Omega rounded to f32, FP32 values in the products,
and float32 results.  The checker computes in f32 throughout, so results agree
to the checker's own f32 rounding.  lanczos as written (defect D1: ritvec reads
eigenvector entries transposed) turns rounding differences into large changes
of its singular values on most inputs, so LAS2 parity is taken on inputs where
the f32 and f64 checkers agree (a Krylov space exhausted at rank k) and the
tolerance is written per case.  On the other inputs the step count itself
depends on f32 rounding: after k steps on a rank-k matrix startv's
`dot <= eps * rnm2` test (mod.rs:634-637) sees a residual near f32 epsilon
in the checker and near f64 epsilon on the GPU.
"""
import numpy as np
import pytest

import matrices as M
import oracle as O
from gpu_util import upload
from single_svdlib import UnsupportedError, lanczos, randomized
from single_svdlib.randomized import PowerIterationNormalizer as PIN

pytestmark = pytest.mark.gpu

F32_EPS34 = float(np.float32(np.finfo(np.float32).eps) ** np.float32(0.75))


def rank_k(m, n, k, seed, top=100.0):
    """Dense m x n matrix of rank k with singular values geomspace(top, 1, k), f32 values."""
    rng = np.random.default_rng(seed)
    U, _ = np.linalg.qr(rng.standard_normal((m, k)))
    V, _ = np.linalg.qr(rng.standard_normal((n, k)))
    return M.dense(((U * np.geomspace(top, 1, k)) @ V.T).astype(np.float32))


def f32_matrix(A):
    B = dict(A)
    B["data"] = np.asarray(A["data"], dtype=np.float32).astype(np.float64)
    return B


def test_f32_handles_hold_the_f32_values():
    A = f32_matrix(M.uniform(300, 200, 0.05, 3))
    D = M.to_scipy(A).toarray()
    x = np.random.default_rng(1).standard_normal(200)
    y = np.random.default_rng(2).standard_normal(300)
    for kind in ("csr", "csc", "coo"):
        h = upload(kind, A, dtype=np.float32)
        assert h.dtype == np.float32
        np.testing.assert_allclose(h.svd_opa(x), D @ x, rtol=0, atol=1e-12 * np.abs(D @ x).max())
        np.testing.assert_allclose(h.svd_opa(y, transposed=True), D.T @ y, rtol=0, atol=1e-12 * np.abs(D.T @ y).max())
    mv = upload("masked", A, mask=(np.arange(200) % 3 != 0).astype(np.uint8), dtype=np.float32)
    assert mv.dtype == np.float32


@pytest.mark.parametrize("case,dims,seed,s_tol", [
    ("rank6_120x80", 3, 3, 1e-4),
    ("rank6_120x80", 5, 3, 1e-4),
    ("rank5_90x150", 3, 3, 1e-4),
    ("rank6_100x160", 3, 11, 1e-4),
    ("dense_30x20", 5, 3, 2e-3),
])
def test_lanczos_f32_parity_with_f32_checker(case, dims, seed, s_tol):
    A = {"rank6_120x80": lambda: rank_k(120, 80, 6, 1), "rank5_90x150": lambda: rank_k(90, 150, 5, 2),
         "rank6_100x160": lambda: rank_k(100, 160, 6, 5),
         "dense_30x20": lambda: f32_matrix(M.uniform(30, 20, 1.0, 1))}[case]()
    ref = O.las2("csr", A, dims, 0, seed=seed, scalar="f32")
    got = lanczos.las2_traced(upload("csr", A, dtype=np.float32), dims, 0, random_seed=seed)
    assert got["error"] is None, got["error"]
    rec = got["rec"]
    dg = rec.diagnostics
    assert rec.s.dtype == np.float32 and rec.u.dtype == np.float32 and rec.vt.dtype == np.float32
    assert rec.d == ref["d"]
    assert dg.lanczos_steps == ref["diagnostics"]["lanczos_steps"]
    assert dg.ritz_values_stabilized == ref["diagnostics"]["ritz_values_stabilized"]
    assert dg.transposed == ref["diagnostics"]["transposed"]
    # kappa is clamped to f32 eps34 (mod.rs:162) and reported as f32
    assert dg.kappa == pytest.approx(F32_EPS34, rel=1e-7)
    assert dg.kappa == ref["diagnostics"]["kappa"]
    # the first step runs on the f32 start vector: alpha_0 as in the f32 checker
    np.testing.assert_allclose(got["alf"][0], ref["alf"][0], rtol=1e-5)
    # converged Ritz values of the last analysis
    k = dg.ritz_values_stabilized
    np.testing.assert_allclose(np.sort(got["ritz"])[-k:], np.sort(ref["ritz"])[-k:], rtol=1e-5,
                               atol=1e-5 * np.abs(ref["ritz"]).max())
    np.testing.assert_allclose(rec.s, ref["s"], rtol=0, atol=s_tol * ref["s"].max())


def test_lanczos_f32_entry_points_and_limits():
    A = rank_k(120, 80, 6, 1)
    h = upload("csr", A, dtype=np.float32)
    r1 = lanczos.svd_dim_seed(h, 4, 3)
    r2 = lanczos.svd_las2(h, 4, 0, (-1e-30, 1e-30), 1e-6, 3)
    np.testing.assert_array_equal(r1.s, r2.s)
    assert r1.s.dtype == np.float32 and r1.u.shape == (4, 120) and r1.vt.shape == (4, 80)
    assert lanczos.svd(h).s.dtype == np.float32
    out = lanczos.las2_traced(h, 4, 0, random_seed=3, algorithm="legacy")
    assert isinstance(out["error"], UnsupportedError)  # legacy::svdLAS2 is f64-only in the crate


@pytest.mark.parametrize("norm", ["QR", "LU"])
@pytest.mark.parametrize("mean_center", [False, True])
def test_randomized_f32_parity_with_f32_checker(norm, mean_center):
    A = f32_matrix(M.lowrank_plus_noise(500, 160, 12, 1e-2, 31, density=0.3))
    om = M.omega(160, 18, 5)
    ref = O.randomized(A, 10, 8, 2, norm, omega=om, mean_center=mean_center, scalar="f32")
    ref64 = O.randomized(A, 10, 8, 2, norm, omega=np.float32(om).astype(np.float64), mean_center=mean_center)
    got = randomized.randomized_svd(upload("csr", A, dtype=np.float32), 10, 8, 2, getattr(PIN, norm), mean_center,
                                    7, False, omega=om)
    assert got.s.dtype == np.float32 and got.u.shape == (500, 10) and got.vt.shape == (10, 160)
    # the f32 checker's own error against the f64 checker on the same f32 inputs bounds the agreement
    own = np.max(np.abs(ref["s"] - ref64["s"]) / ref64["s"])
    rel = np.max(np.abs(got.s - ref["s"]) / ref["s"])
    assert rel < max(4 * own, 2e-6), (rel, own)
    rel64 = np.max(np.abs(got.s.astype(np.float64) - ref64["s"]) / ref64["s"])
    assert rel64 < 2e-6, rel64
