"""randomized::* (src/randomized/mod.rs): randomized SVD on the GPU."""
from __future__ import annotations

import ctypes as C
import enum

import numpy as np

from . import _abi
from ._core import SvdRec, as_smat, check, options, rec_from_c


class PowerIterationNormalizer(enum.Enum):
    """PowerIterationNormalizer (mod.rs:14-19)."""

    QR = "QR"
    LU = "LU"
    None_ = "None"


def randomized_svd(m, target_rank, n_oversamples, n_power_iters, power_iteration_normalizer=PowerIterationNormalizer.QR,
                   mean_center=False, seed=None, verbose=False, precision="f64", omega=None) -> SvdRec:
    """randomized::randomized_svd (mod.rs:24-199).

    ``omega`` (ncols x (rank + n_oversamples), row-major) fixes the Gaussian
    test matrix; otherwise it is drawn on the device from ``seed``.
    """
    a = as_smat(m)
    norm = power_iteration_normalizer
    if isinstance(norm, PowerIterationNormalizer):
        norm = norm.value
    om = None if omega is None else np.ascontiguousarray(omega, dtype=np.float64)
    o = options(precision=precision, verbose=verbose, omega=om)
    r = _abi.svdb_rec()
    try:
        check(_abi.lib().svdb_randomized_svd(a.handle, target_rank, n_oversamples, n_power_iters,
                                             _abi.NORMALIZER[norm], int(mean_center), int(seed is not None),
                                             0 if seed is None else int(seed), int(verbose), C.byref(o),
                                             C.byref(r)))
        return rec_from_c(r)
    finally:
        _abi.lib().svdb_rec_free(C.byref(r))


def svd_flip(u=None, v=None, u_based_decision=True):
    """randomized::svd_flip (mod.rs:332-438) on copies of u (m x k) and v (k x n); returns (u, v).

    Runs on the GPU (svdb_svd_flip).  Missing inputs raise Las2Error as the crate does.
    """
    uu = None if u is None else np.array(u, dtype=np.float64, order="C", copy=True)
    vv = None if v is None else np.array(v, dtype=np.float64, order="C", copy=True)
    ur, uc = (0, 0) if uu is None else uu.shape
    vr, vc = (0, 0) if vv is None else vv.shape
    check(_abi.lib().svdb_svd_flip(None if uu is None else uu.ctypes.data, ur, uc,
                                   None if vv is None else vv.ctypes.data, vr, vc, int(u_based_decision), 0))
    return uu, vv
