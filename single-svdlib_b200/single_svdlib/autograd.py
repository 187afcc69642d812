"""torch.autograd harness around the truncated SVD of a sparse matrix.

``TruncatedSVD.apply(values, indptr, indices, shape, k, method, seed, cg_tol, power_iters)``
returns U (m x k), s (k), V (n x k) of the CSR matrix with the given values
(float64 torch tensors, signs fixed by svd_flip on U), and its backward
returns dL/dvalues through ``svdb_svd_adjoint`` (block CG + SDDMM on the
GPU).  torch is only the autograd plumbing; every product runs in
libsvdb200.so.
"""
from __future__ import annotations

import numpy as np
import torch

from . import adjoint as _adj
from . import legacy as _legacy
from . import randomized as _rand
from ._core import CsrMatrix


def _forward_svd(mat, k, method, seed, power_iters):
    if method == "randomized":
        rec = _rand.randomized_svd(mat, k, max(10, k), power_iters, _rand.PowerIterationNormalizer.QR, False, seed,
                                   False)
        u, s, vt = rec.u, rec.s, rec.vt            # u: m x d
    elif method == "las2":
        rec = _legacy.svd_las2(mat, k, 0, (-1e-30, 1e-30), 1e-12, seed)
        u, s, vt = rec.ut.T, rec.s, rec.vt          # legacy ut: d x m
    else:
        raise ValueError(f"unknown method {method!r}")
    if rec.d < k:
        raise RuntimeError(f"truncated SVD found {rec.d} of {k} triplets")
    u, vt = _rand.svd_flip(u[:, :k], vt[:k], True)
    return u, np.ascontiguousarray(s[:k]), np.ascontiguousarray(vt.T)


class TruncatedSVD(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values, indptr, indices, shape, k, method="randomized", seed=7, cg_tol=1e-12, power_iters=20):
        vals = values.detach().cpu().numpy().astype(np.float64)
        mat = CsrMatrix(shape[0], shape[1], np.asarray(indptr), np.asarray(indices), vals)
        u, s, v = _forward_svd(mat, k, method, seed, power_iters)
        ctx.mat = mat
        ctx.cg_tol = cg_tol
        ctx.values_device = values.device
        U, S, V = (torch.from_numpy(x) for x in (u, s, v))
        ctx.save_for_backward(U, S, V)
        return U.to(values.device), S.to(values.device), V.to(values.device)

    @staticmethod
    def backward(ctx, gU, gs, gV):
        U, S, V = ctx.saved_tensors

        def host(g):
            return None if g is None else g.detach().cpu().numpy().astype(np.float64)

        grad = _adj.svd_adjoint(ctx.mat, U.numpy(), S.numpy(), V.numpy(), host(gU), host(gs), host(gV),
                                cg_tol=ctx.cg_tol)
        ctx.mat.close()
        return torch.from_numpy(grad).to(ctx.values_device), None, None, None, None, None, None, None, None


def truncated_svd(values, indptr, indices, shape, k, method="randomized", seed=7, cg_tol=1e-12, power_iters=20):
    """U, s, V of the k leading singular triplets; differentiable in ``values``.

    The randomized forward's error falls as (s_{k+11} / s_k)^(2 power_iters + 1);
    finite-difference checks need it near machine precision."""
    return TruncatedSVD.apply(values, indptr, indices, shape, k, method, seed, cg_tol, power_iters)
