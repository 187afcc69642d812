"""Adjoint of the truncated SVD with respect to a sparse matrix's stored values.

No counterpart in the crate.  ``svd_adjoint`` returns dL/dvalues for a loss
L(U, s, V) of the k leading singular triplets of A, evaluated only at A's
nonzeros (an SDDMM on the device); the dense gradient it samples is

    U M V^T + Gamma V^T + U Delta^T,

with M the in-subspace term (the F-matrix 1/(s_j^2 - s_i^2)) and (Gamma,
Delta) the complement terms, solved by block CG against A - U S V^T on the
GPU (see include/svdb200.h, svdb_svd_adjoint).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._core import check


@dataclass
class AdjointInfo:
    cg_iterations: int
    cg_residual: float
    time_ms_solve: float
    time_ms_sddmm: float


def _opts(precision, cg_tol, cg_max_iters, on_device=False):
    o = _abi.svdb_adjoint_options()
    _abi.lib().svdb_adjoint_options_default(C.byref(o))
    o.precision = _abi.PRECISION[precision]
    o.inputs_on_device = int(on_device)
    if cg_tol is not None:
        o.cg_tol = float(cg_tol)
    if cg_max_iters is not None:
        o.cg_max_iters = int(cg_max_iters)
    return o


def _arr(x, shape):
    if x is None:
        return None
    a = np.ascontiguousarray(x, dtype=np.float64)
    if a.shape != shape:
        raise ValueError(f"expected shape {shape}, got {a.shape}")
    return a


def svd_adjoint(a, u, s, v, g_u=None, g_s=None, g_v=None, precision="f64", cg_tol=None, cg_max_iters=None,
                return_info=False):
    """dL/dvalues of A (a CsrMatrix or CscMatrix handle), in the handle's entry order.

    u: m x k, s: k, v: n x k (the k leading triplets, s descending);
    g_u, g_s, g_v: dL/du, dL/ds, dL/dv (None = 0).  Other handle kinds raise
    UnsupportedError from the library.
    """
    m, n = a.shape
    s = np.ascontiguousarray(s, dtype=np.float64).ravel()
    k = s.shape[0]
    u = _arr(u, (m, k))
    v = _arr(v, (n, k))
    g_u = _arr(g_u, (m, k))
    g_v = _arr(g_v, (n, k))
    g_s = None if g_s is None else _arr(np.ravel(g_s), (k,))
    out = np.empty(a.nnz(), dtype=np.float64)
    o = _opts(precision, cg_tol, cg_max_iters)

    def p(x):
        return None if x is None else x.ctypes.data

    check(_abi.lib().svdb_svd_adjoint(a.handle, k, p(u), p(s), p(v), p(g_u), p(g_s), p(g_v), C.byref(o),
                                      out.ctypes.data))
    info = AdjointInfo(int(o.cg_iterations), float(o.cg_residual), float(o.time_ms_solve), float(o.time_ms_sddmm))
    return (out, info) if return_info else out


def sddmm_device(a, left_ptr, right_ptr, rank, out_ptr, precision="f64", stream=None):
    """out[e] = left[r_e] . right[c_e] on device buffers (float for 'mixed', double for 'f64')."""
    check(_abi.lib().svdb_sddmm_device(a.handle, left_ptr, right_ptr, rank, out_ptr, _abi.PRECISION[precision],
                                       stream))
