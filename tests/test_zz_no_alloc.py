"""svdb_opb_device_noalloc: the operator A^T A x for callers that cannot
allocate device memory (their allocator holds the GPU, or an allocation's
synchronisation is not acceptable where they call).  Its intermediate vector
lives in a fixed 8 MiB array inside the library.

Checked through the C ABI against svdb_opb, the allocating entry point, with
the 1e-13 relative tolerance of the other operator tests, on two calls in a
row (the shared array keeps the previous call's contents).  Collected last so
that a run stopping at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import matrices as M
from single_svdlib import CsrMatrix, _abi

pytestmark = pytest.mark.gpu


def _noalloc(h, x, transposed):
    import torch
    out_len = h.nrows() if transposed else h.ncols()
    dx = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    dy = torch.full((out_len,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = _abi.lib().svdb_opb_device_noalloc(h.handle, dx.data_ptr(), dy.data_ptr(), int(transposed), None)
    assert rc == 0, _abi.last_error()
    torch.cuda.synchronize()
    return dy.cpu().numpy()


def _close(a, b):
    np.testing.assert_allclose(a, b, rtol=0, atol=1e-13 * max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("transposed", [False, True])
def test_matches_svdb_opb_on_two_calls(transposed):
    rng = np.random.default_rng(17)
    A1 = M.uniform(3000, 1200, 0.01, 3)
    A2 = M.poisson_rows(700, 2500, 9, 4)  # a second, smaller operator: stale scratch must not leak in
    for A in (A1, A2):
        h = CsrMatrix(A["nrows"], A["ncols"], A["indptr"], A["indices"], A["data"])
        n_in = A["nrows"] if transposed else A["ncols"]
        for _ in range(2):
            x = rng.standard_normal(n_in)
            _close(_noalloc(h, x, transposed), h.svd_opb(x, transposed=transposed))


def test_first_call_allocates_nothing():
    """The device's free memory is the same before and after the first call on
    a fresh handle: the scratch array was placed when the handle was created."""
    import torch
    A = M.uniform(2000, 900, 0.01, 5)
    h = CsrMatrix(A["nrows"], A["ncols"], A["indptr"], A["indices"], A["data"])
    x = np.random.default_rng(3).standard_normal(A["ncols"])
    want = h.svd_opb(x)  # the allocating path loads the same SpMV kernel
    dx = torch.from_numpy(x).cuda()
    dy = torch.zeros(A["ncols"], dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    rc = _abi.lib().svdb_opb_device_noalloc(h.handle, dx.data_ptr(), dy.data_ptr(), 0, None)
    assert rc == 0, _abi.last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    _close(dy.cpu().numpy(), want)


def test_rejects_intermediates_above_the_limit():
    import scipy.sparse as sp
    m = (1 << 20) + 1
    S = sp.csr_matrix((np.ones(4), ([0, 5, 1000, m - 1], [0, 1, 2, 3])), shape=(m, 4))
    A = M.from_scipy(S)
    h = CsrMatrix(A["nrows"], A["ncols"], A["indptr"], A["indices"], A["data"])
    import torch
    dx = torch.ones(4, dtype=torch.float64, device="cuda")
    dy = torch.zeros(4, dtype=torch.float64, device="cuda")
    rc = _abi.lib().svdb_opb_device_noalloc(h.handle, dx.data_ptr(), dy.data_ptr(), 0, None)
    assert rc == 9 and "exceeds the fixed scratch" in _abi.last_error()
