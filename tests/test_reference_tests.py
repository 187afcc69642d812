"""The crate's own behaviour tests (src/lib.rs:111-280), on the matrices its
generators make (tests/rand_restate.py restates them; bit identity with the
rand crates is unverified, see there):

- test_real_sparse_matrix (src/lib.rs:156-164): lanczos::svd_dim_seed, as
  written, on the 100 x 100 COO of density 0.98 %, dimensions 50, seed 42,
  returns Ok.  This and the next are the reference-held behaviour pins of the
  as-written LAS2 path, the drop-in default.
- random_matrix_comparison (src/lib.rs:111-154): on the 50 x 30 CSR from 300
  random pushes (repeats summed) with seed 12345, svd_dim_seed(.., 0, 12345)
  on the CSR and on MaskedCSRMatrix::new with every column give the same
  rank and singular values within 1e-3 relative.
- test_random_svd_computation / test_randomized_svd_small_sparse_matrix
  (src/lib.rs:165-280): randomized_svd(csr of the 1000 x 250 COO of density
  1 %, 50, 10, 3 or 2, QR, no centring, seed 42) succeeds with d = 50 and
  positive, descending singular values.  (The crate itself stops in todo!()
  on a plain CsrMatrix here, src/lanczos/mod.rs:1629-1654; the library runs
  it.  u is m x d for randomized_svd, as the crate's code returns it,
  src/randomized/mod.rs:175-184, not the d x m the crate's test asserts.)

Each runs on the checker (CPU) and, marked gpu, through the library.
"""
import numpy as np
import pytest

import oracle as O
import rand_restate as R
from single_svdlib import CooMatrix, CsrMatrix, MaskedCSRMatrix, lanczos, randomized
from single_svdlib.randomized import PowerIterationNormalizer as PIN


@pytest.fixture(scope="module")
def real_sparse():
    return R.create_sparse_matrix(100, 100, 0.0098)


@pytest.fixture(scope="module")
def comparison():
    return R.coo_to_csr(R.random_coo(50, 30, 12345))


def test_generators_are_the_crates_shape(real_sparse, comparison):
    A = real_sparse
    assert len(A["data"]) == 98 and len(set(zip(A["row"], A["col"]))) == 98
    assert np.all(np.abs(A["data"]) > 1e-10) and np.all(np.abs(A["data"]) < 10.0)
    assert A["row"].max() < 100 and A["col"].max() < 100
    C = comparison
    assert C["nrows"] == 50 and C["ncols"] == 30 and 250 <= len(C["data"]) <= 300
    # the stream is deterministic
    np.testing.assert_array_equal(R.create_sparse_matrix(100, 100, 0.0098)["data"], A["data"])


def test_real_sparse_matrix_checker(real_sparse):
    r = O.las2("coo", real_sparse, 50, 0, seed=42, legacy=False)
    assert r["d"] >= 1 and np.all(np.isfinite(r["s"]))


def test_random_matrix_comparison_checker(comparison):
    a = O.las2("csr", comparison, 0, 0, seed=12345, legacy=False)
    b = O.las2("masked", comparison, 0, 0, seed=12345, legacy=False, mask=np.ones(30, np.uint8))
    assert a["d"] == b["d"]
    np.testing.assert_allclose(b["s"], a["s"], rtol=1e-3)


@pytest.mark.gpu
def test_real_sparse_matrix(real_sparse):
    A = real_sparse
    rec = lanczos.svd_dim_seed(CooMatrix(100, 100, A["row"], A["col"], A["data"]), 50, 42)
    ref = O.las2("coo", A, 50, 0, seed=42, legacy=False)
    assert rec.d == ref["d"] and rec.diagnostics.lanczos_steps == ref["diagnostics"]["lanczos_steps"]
    assert np.all(np.isfinite(rec.s))


@pytest.mark.gpu
def test_random_matrix_comparison(comparison):
    C = comparison
    csr = CsrMatrix(50, 30, C["indptr"], C["indices"], C["data"])
    plain = lanczos.svd_dim_seed(csr, 0, 12345)
    masked = lanczos.svd_dim_seed(MaskedCSRMatrix(csr, np.ones(30, bool)), 0, 12345)
    assert plain.d == masked.d
    for a, b in zip(plain.s, masked.s):
        assert abs(a - b) / max(a, b) <= 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("q", [3, 2])
def test_random_svd_computation(q):
    A = R.coo_to_csr(R.create_sparse_matrix(1000, 250, 0.01))
    csr = CsrMatrix(1000, 250, A["indptr"], A["indices"], A["data"])
    rec = randomized.randomized_svd(csr, 50, 10, q, PIN.QR, False, 42, False)
    assert rec.d == 50
    assert np.all(rec.s > 0) and np.all(np.diff(rec.s) <= 0)
    assert rec.u.shape == (1000, 50) and rec.vt.shape == (50, 250)
