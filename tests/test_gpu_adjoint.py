"""Adjoint of the truncated SVD (svdb_svd_adjoint) and its SDDMM, svd_flip.

The adjoint is checked three ways: against torch's dense SVD backward on
small matrices (feeding torch's own triplets, so only the adjoint is
tested), against f64 central finite differences of the whole GPU pipeline
(forward randomized SVD + svd_flip, backward adjoint) on a matrix with a
clear spectral gap, and its SDDMM against numpy.  Tolerances: 1e-8 of the
largest gradient entry against the dense reference; 1e-6 against central
finite differences of step 1e-4 (and 1e-4 at step 1e-6, the f64 rounding
floor of that step)."""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

import matrices as M
import oracle as O
from gpu_util import upload
from single_svdlib import CooMatrix, CscMatrix, CsrMatrix, UnsupportedError, adjoint, randomized
from single_svdlib._core import Las2Error
from single_svdlib.autograd import truncated_svd

pytestmark = pytest.mark.gpu


def dense_reference(A, k, gU, gs, gV):
    """torch f64: triplets of the dense thin SVD and dL/dA of
    L = <gU, U_k> + <gs, s_k> + <gV, V_k>."""
    At = torch.tensor(M.to_scipy(A).toarray(), dtype=torch.float64, requires_grad=True)
    U, S, Vh = torch.linalg.svd(At, full_matrices=False)
    Uk, Sk, Vk = U[:, :k], S[:k], Vh[:k].T
    loss = (torch.from_numpy(gU) * Uk).sum() + (torch.from_numpy(gs) * Sk).sum() + (torch.from_numpy(gV) * Vk).sum()
    loss.backward()
    return Uk.detach().numpy(), Sk.detach().numpy(), Vk.detach().numpy(), At.grad.numpy()


def at_pattern(A, D):
    rows = np.repeat(np.arange(A["nrows"]), np.diff(A["indptr"]))
    return D[rows, A["indices"]]


@pytest.mark.parametrize("shape,k", [((70, 45), 5), ((40, 90), 6), ((120, 120), 8)])
def test_adjoint_matches_dense_backward(shape, k):
    m, n = shape
    A = M.uniform(m, n, 0.25, 100 + m, -1.0, 1.0)
    rng = np.random.default_rng(5)
    gU, gs, gV = rng.standard_normal((m, k)), rng.standard_normal(k), rng.standard_normal((n, k))
    U, S, V, D = dense_reference(A, k, gU, gs, gV)
    got, info = adjoint.svd_adjoint(upload("csr", A), U, S, V, gU, gs, gV, return_info=True)
    ref = at_pattern(A, D)
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() <= 1e-8 * scale, (np.abs(got - ref).max(), scale, info)
    assert info.cg_residual <= 1e-12


def test_adjoint_partial_cotangents_and_csc_order():
    A = M.uniform(60, 50, 0.3, 7, -1.0, 1.0)
    k = 4
    rng = np.random.default_rng(9)
    gU, gs, gV = rng.standard_normal((60, k)), np.zeros(k), np.zeros((50, k))
    U, S, V, D = dense_reference(A, k, gU, gs, gV)
    # only g_u given; the others are None
    got = adjoint.svd_adjoint(upload("csr", A), U, S, V, g_u=gU)
    np.testing.assert_allclose(got, at_pattern(A, D), rtol=0, atol=1e-8 * np.abs(D).max())
    # CSC handle: gradient in CSC entry order
    C = M.to_csc(A)
    h = CscMatrix(C["nrows"], C["ncols"], C["indptr"], C["indices"], C["data"])
    got_c = adjoint.svd_adjoint(h, U, S, V, g_u=gU)
    cols = np.repeat(np.arange(C["ncols"]), np.diff(C["indptr"]))
    np.testing.assert_allclose(got_c, D[C["indices"], cols], rtol=0, atol=1e-8 * np.abs(D).max())


def test_adjoint_singular_value_only_is_uv_outer():
    # dL/dA for L = <gs, s> is U diag(gs) V^T: no solve needed beyond CG's first residual
    A = M.uniform(50, 40, 0.4, 3, -1.0, 1.0)
    k = 3
    d = M.to_scipy(A).toarray()
    U, S, Vt = np.linalg.svd(d, full_matrices=False)
    gs = np.array([1.0, -2.0, 0.5])
    got = adjoint.svd_adjoint(upload("csr", A), U[:, :k], S[:k], Vt[:k].T, g_s=gs)
    ref = at_pattern(A, (U[:, :k] * gs) @ Vt[:k])
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12 * np.abs(ref).max())


def gap_matrix(m, n, density, seed, amps=(6.0, 5.0, 4.0, 3.5)):
    """N(0,1) values plus a constant on each of len(amps) diagonal blocks, at a
    random pattern: block constants survive the sampling, so the spectrum has
    a gap after len(amps) (s_5 / s_4 = 0.46 for the case below)."""
    rng = np.random.default_rng(seed)
    mask = rng.random((m, n)) < density
    D = rng.standard_normal((m, n))
    rb, cb = m // len(amps), n // len(amps)
    for i, c in enumerate(amps):
        D[i * rb:(i + 1) * rb, i * cb:(i + 1) * cb] += c
    return M.from_scipy(sp.csr_matrix(np.where(mask, D, 0.0)))


def test_adjoint_finite_differences_through_autograd():
    A = gap_matrix(300, 200, 0.5, 21)
    k = 4
    s_all = np.linalg.svd(M.to_scipy(A).toarray(), compute_uv=False)
    assert s_all[k] / s_all[k - 1] < 0.5  # the planted gap
    rng = np.random.default_rng(11)
    gU, gs, gV = rng.standard_normal((300, k)), rng.standard_normal(k), rng.standard_normal((200, k))
    tU, tgs, tV = (torch.from_numpy(x) for x in (gU, gs, gV))
    indptr, indices = A["indptr"], A["indices"]

    def loss_of(vals):
        U, S, V = truncated_svd(vals, indptr, indices, (300, 200), k, "randomized", 3)
        return (tU * U).sum() + (tgs * S).sum() + (tV * V).sum()

    vals = torch.tensor(A["data"], dtype=torch.float64, requires_grad=True)
    loss = loss_of(vals)
    loss.backward()
    g = vals.grad.numpy()
    picks = rng.choice(len(A["data"]), 25, replace=False)
    # Central differences: at step 1e-4 the truncation error is ~1e-8 of the
    # gradient here; at the step 1e-6 the f64 forward's rounding (~1e-15 |L|)
    # over 2h already reaches ~1e-5 of the largest entry (an exact LAPACK
    # forward gives 1.6e-5), so that step is held to its rounding floor.
    for h, tol in ((1e-4, 1e-6), (1e-6, 1e-4)):
        fd = []
        for e in picks:
            vp = A["data"].copy(); vp[e] += h
            vm = A["data"].copy(); vm[e] -= h
            with torch.no_grad():
                fp = loss_of(torch.from_numpy(vp)).item()
                fm = loss_of(torch.from_numpy(vm)).item()
            fd.append((fp - fm) / (2 * h))
        fd = np.array(fd)
        err = np.abs(fd - g[picks]).max() / np.abs(g[picks]).max()
        assert err <= tol, (h, err, fd[:5], g[picks][:5])


@pytest.mark.parametrize("rank", [1, 24, 64, 100])
@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_sddmm_device(rank, precision):
    # long rows (several segments), empty rows, ragged rank
    rng = np.random.default_rng(rank)
    D = (rng.random((300, 6000)) < 0.02) * rng.standard_normal((300, 6000))
    D[5, :] = rng.standard_normal(6000)   # 6000 entries: 3 segments
    D[7, :] = 0.0
    A = M.from_scipy(sp.csr_matrix(D))
    L, R = rng.standard_normal((300, rank)), rng.standard_normal((6000, rank))
    ref = O.sddmm(A, L, R)
    h = upload("csr", A)
    dt = torch.float64 if precision == "f64" else torch.float32
    tl, tr = torch.tensor(L, dtype=dt, device="cuda"), torch.tensor(R, dtype=dt, device="cuda")
    out = torch.empty(len(A["data"]), dtype=dt, device="cuda")
    adjoint.sddmm_device(h, tl.data_ptr(), tr.data_ptr(), rank, out.data_ptr(), precision)
    torch.cuda.synchronize()
    got = out.double().cpu().numpy()
    tol = 1e-12 if precision == "f64" else 1e-5
    assert np.abs(got - ref).max() <= tol * max(1.0, np.abs(ref).max()) * np.sqrt(rank)


def test_adjoint_errors():
    A = M.uniform(30, 20, 0.3, 1, -1.0, 1.0)
    C = M.to_coo(A)
    coo = CooMatrix(C["nrows"], C["ncols"], C["row"], C["col"], C["data"])
    U, S, V = np.ones((30, 2)), np.array([2.0, 1.0]), np.ones((20, 2))
    with pytest.raises(UnsupportedError):
        adjoint.svd_adjoint(coo, U, S, V)
    with pytest.raises(ValueError):
        adjoint.svd_adjoint(upload("csr", A), U, np.array([1.0, 0.0]), V)
    out = adjoint.svd_adjoint(upload("csr", A), np.zeros((30, 0)), np.zeros(0), np.zeros((20, 0)))
    assert out.shape == (len(A["data"]),) and not out.any()


@pytest.mark.parametrize("u_based", [True, False])
def test_svd_flip_matches_checker(u_based):
    rng = np.random.default_rng(4)
    u = rng.standard_normal((50, 6))
    v = rng.standard_normal((6, 40))
    u[:, 2] = 0.0               # all-zero column decides by entry 0
    u[3, 4], u[9, 4] = -5.0, 5.0  # tie: the first one decides
    v[1, 7], v[1, 2] = 7.0, -7.0
    gu, gv = randomized.svd_flip(u, v, u_based)
    ru, rv = O.svd_flip(u, v, u_based)
    np.testing.assert_array_equal(gu, ru)
    np.testing.assert_array_equal(gv, rv)
    # mismatched counts: only the common leading vectors are flipped on the other side
    gu2, gv2 = randomized.svd_flip(u, v[:4], u_based)
    ru2, rv2 = O.svd_flip(u, v[:4], u_based)
    np.testing.assert_array_equal(gu2, ru2)
    np.testing.assert_array_equal(gv2, rv2)


def test_svd_flip_errors():
    with pytest.raises(Las2Error):
        randomized.svd_flip(None, None)
    with pytest.raises(Las2Error):
        randomized.svd_flip(None, np.ones((2, 2)), True)
    with pytest.raises(Las2Error):
        randomized.svd_flip(np.ones((2, 2)), None, False)
