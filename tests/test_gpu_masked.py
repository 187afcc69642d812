"""MaskedCSRMatrix on the GPU: the column remap and compaction are integer
work and must be bit-exact (src/lanczos/masked.rs:21-102)."""
import numpy as np
import pytest

import matrices as M
import oracle as O
from single_svdlib import CsrMatrix, MaskedCSRMatrix, ShapeError

pytestmark = pytest.mark.gpu


def csr(A):
    return CsrMatrix(A["nrows"], A["ncols"], A["indptr"], A["indices"], A["data"])


@pytest.mark.parametrize("p", [0.0, 0.01, 0.5, 0.99, 1.0])
def test_maps_and_nnz_bit_exact(p):
    A = M.uniform(500, 3000, 0.01, 8)
    mask = (np.random.default_rng(9).random(3000) < p).astype(np.uint8)
    parent = csr(A)
    mv = MaskedCSRMatrix(parent, mask)
    m2o, o2m, mnnz = O.masked_maps(A, mask)
    g_m2o, g_o2m = mv.maps()
    assert np.array_equal(g_m2o, m2o)
    assert np.array_equal(g_o2m, o2m)
    assert mv.nnz() == mnnz
    assert mv.ncols() == len(m2o) and mv.nrows() == 500
    assert mv.uses_all_columns() == (p == 1.0)


def test_with_columns_dedup_and_order():  # masked.rs:48-55
    A = M.uniform(40, 30, 0.2, 1)
    parent = csr(A)
    v = MaskedCSRMatrix.with_columns(parent, [7, 3, 3, 29, 0])
    assert list(v.maps()[0]) == [0, 3, 7, 29]


def test_3x5_known_answer():  # masked.rs:885-907
    import scipy.sparse as sp
    S = sp.csr_matrix(([1, 2, 3, 4, 5, 6, 7, 8], ([0, 0, 0, 1, 1, 2, 2, 2], [0, 2, 4, 1, 3, 0, 2, 4])), shape=(3, 5))
    v = MaskedCSRMatrix.with_columns(csr(M.from_scipy(S)), [0, 2, 4])
    assert (v.nrows(), v.ncols(), v.nnz()) == (3, 3, 6)


def test_shape_errors():
    parent = csr(M.uniform(10, 8, 0.3, 2))
    with pytest.raises(ShapeError, match="same length"):
        MaskedCSRMatrix(parent, np.ones(7, np.uint8))
    with pytest.raises(ShapeError, match="out of bounds"):
        MaskedCSRMatrix.with_columns(parent, [1, 8])


def test_large_masked_compaction():
    A = M.poisson_rows(20000, 30000, 50, 13)
    mask = (np.random.default_rng(14).random(30000) < 0.3).astype(np.uint8)
    mv = MaskedCSRMatrix(csr(A), mask)
    m2o, o2m, mnnz = O.masked_maps(A, mask)
    assert mv.nnz() == mnnz
    assert np.array_equal(mv.maps()[0], m2o)
    # the compacted operator equals the physical column subset
    S = M.to_scipy(A)[:, m2o]
    x = np.random.default_rng(3).standard_normal(len(m2o))
    np.testing.assert_allclose(mv.svd_opa(x), S @ x, rtol=0, atol=1e-12 * np.abs(S @ x).max())


def test_view_then_parent_teardown_after_mixed_precision():
    # the FP32 copy made through an all-columns view belongs to the parent and must
    # outlive the view's stream
    from single_svdlib import randomized
    from single_svdlib.randomized import PowerIterationNormalizer as PIN
    A = M.uniform(300, 100, 0.1, 61)
    parent = csr(A)
    mv = MaskedCSRMatrix(parent, np.ones(100, np.uint8))
    r = randomized.randomized_svd(mv, 5, 5, 1, PIN.QR, False, 1, False, precision="mixed")
    assert r.d == 5
    mv.close()
    parent.close()
