"""Failure paths, tested without faulting or hanging the GPU.

- Bounded device waits: the library's grid barrier and mbarrier wait are made
  to run out on purpose (a second arrival that never comes; a barrier nothing
  arrives on) through svdb_wait_selftest, which must return SVDB_ERR_TIMEOUT
  after about its limit and leave the context usable.
- The same limit on a real solve: with SVDB_WAIT_LIMIT_NS=1 the cooperative
  Lanczos block (grid mode) gives up at a barrier where a block has to wait,
  and the call returns SVDB_ERR_TIMEOUT; the next solve on a fresh handle, at
  the normal limit, matches the checker.
- Corrupt compressed input: offsets that do not start at 0, do not end at
  nnz, or fall; an index at or past the minor dimension.  Each is refused with
  SVDB_ERR_SHAPE, as the crate's constructors refuse them
  (nalgebra-sparse's CsrMatrix::try_from_csr_data, used by the crate's tests,
  src/lib.rs:22-60), and the next upload works.
"""
import time

import numpy as np
import pytest

import matrices as M
import oracle as O
from gpu_util import upload
from single_svdlib import CooMatrix, CscMatrix, CsrMatrix, DeviceError, ShapeError, _abi, legacy

pytestmark = pytest.mark.gpu

TIMEOUT = 8


@pytest.mark.parametrize("which", [0, 1])
def test_bounded_wait_gives_up_after_its_limit(which):
    L = _abi.lib()
    t0 = time.perf_counter()
    rc = L.svdb_wait_selftest(which, 2_000_000)  # 2 ms
    dt = time.perf_counter() - t0
    assert rc == TIMEOUT, (rc, _abi.last_error())
    assert 0.002 <= dt < 1.0, dt
    # the context is still usable: a solve right after matches the checker
    A = M.poisson_rows(300, 120, 6, 9)
    got = legacy.svd_dim_seed(upload("csr", A), 4, 3)
    ref = O.las2("csr", A, 4, 0, seed=3, legacy=True)
    np.testing.assert_allclose(got.s, ref["s"], rtol=1e-10)


def test_selftest_rejects_bad_arguments():
    L = _abi.lib()
    assert L.svdb_wait_selftest(2, 1000) == 10
    assert L.svdb_wait_selftest(0, 0) == 10


def _grid_mode_matrix():
    """Above the cluster threshold (2^20 nonzeros), with a few long rows that
    keep one block busy while the others wait at the next barrier."""
    rng = np.random.default_rng(21)
    m, n = 60_000, 40_000
    lens = rng.poisson(20, m)
    lens[:4] = n  # four full rows
    rows = np.repeat(np.arange(m), lens)
    cols = np.concatenate([rng.choice(n, k, replace=False) for k in lens])
    import scipy.sparse as sp
    S = sp.csr_matrix((rng.random(len(rows)) + 0.1, (rows, cols)), shape=(m, n))
    S.sum_duplicates()
    S.sort_indices()
    return M.from_scipy(S)


def test_lanczos_grid_barrier_limit_returns_timeout(monkeypatch):
    A = _grid_mode_matrix()
    assert len(A["data"]) > (1 << 20)
    monkeypatch.setenv("SVDB_LZ_CLUSTER", "0")
    monkeypatch.setenv("SVDB_WAIT_LIMIT_NS", "1")
    with pytest.raises(DeviceError) as ei:
        legacy.svd_dim_seed(upload("csr", A), 5, 7)
    assert ei.value.status == TIMEOUT and "grid barrier" in str(ei.value)
    monkeypatch.delenv("SVDB_WAIT_LIMIT_NS")
    got = legacy.svd_dim_seed(upload("csr", A), 5, 7)
    ref = O.las2("csr", A, 5, 0, seed=7, legacy=True)
    assert got.diagnostics.lanczos_steps == ref["diagnostics"]["lanczos_steps"]
    np.testing.assert_allclose(got.s, ref["s"], rtol=1e-10)


def _csr_parts():
    A = M.uniform(50, 30, 0.2, 13)
    return A["nrows"], A["ncols"], A["indptr"].copy(), A["indices"].copy(), A["data"].copy()


@pytest.mark.parametrize("defect", ["first", "last", "falling", "index"])
@pytest.mark.parametrize("fmt", ["csr", "csc"])
def test_corrupt_compressed_input_is_refused(defect, fmt):
    m, n, ip, ix, v = _csr_parts()
    major, minor = m, n  # read as a CSC, the same arrays are the transpose (n x m)
    if defect == "first":
        ip[0] = 1
    elif defect == "last":
        ip[-1] = ip[-1] - 1
    elif defect == "falling":
        k = major // 2
        ip[k] = ip[k + 1] + 1
    else:
        ix[len(ix) // 2] = minor
    with pytest.raises(ShapeError) as ei:
        if fmt == "csr":
            CsrMatrix(m, n, ip, ix, v)
        else:
            CscMatrix(n, m, ip, ix, v)
    assert ei.value.status == 6 and "invalid compressed sparse input" in str(ei.value)
    # the next, valid upload works
    m, n, ip, ix, v = _csr_parts()
    h = CsrMatrix(m, n, ip, ix, v)
    x = np.random.default_rng(1).standard_normal(n)
    np.testing.assert_allclose(h.svd_opa(x), M.to_scipy({"nrows": m, "ncols": n, "indptr": ip, "indices": ix,
                                                        "data": v}) @ x, rtol=1e-13)


def test_coo_index_out_of_bounds_is_refused():
    with pytest.raises(ShapeError):
        CooMatrix(5, 4, np.array([0, 1, 5]), np.array([0, 1, 2]), np.ones(3))
    with pytest.raises(ShapeError):
        CooMatrix(5, 4, np.array([0, 1, 2]), np.array([0, 4, 2]), np.ones(3))
