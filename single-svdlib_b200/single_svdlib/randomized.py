"""randomized::* (src/randomized/mod.rs): randomized SVD on the GPU."""
from __future__ import annotations

import ctypes as C
import enum

import numpy as np

from . import _abi
from ._core import ShapeError, SvdRec, as_smat, check, options, rec_from_c


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
    f32 = a.dtype == np.float32  # T = f32: float32 results, precision ignored
    r = _abi.svdb_rec_f32() if f32 else _abi.svdb_rec()
    fn = _abi.lib().svdb_randomized_svd_f32 if f32 else _abi.lib().svdb_randomized_svd
    try:
        check(fn(a.handle, target_rank, n_oversamples, n_power_iters, _abi.NORMALIZER[norm], int(mean_center),
                 int(seed is not None), 0 if seed is None else int(seed), int(verbose), C.byref(o), C.byref(r)))
        return rec_from_c(r)
    finally:
        (_abi.lib().svdb_rec_f32_free if f32 else _abi.lib().svdb_rec_free)(C.byref(r))


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


class RandomizedBatch:
    """randomized_svd on many MaskedCSRMatrix::with_columns subsets of one matrix.

    ``subsets`` is a sequence of column lists (with_columns semantics: order and
    duplicates ignored).  The batch is prepared once (maps, workspaces, the
    autotuned product shape and the captured CUDA graph); ``run()`` replays it
    and returns one SvdRec per subset, each as randomized_svd(masked_b, ...)
    with the same seed would.
    """

    def __init__(self, matrix, subsets, target_rank, n_oversamples, n_power_iters,
                 power_iteration_normalizer=PowerIterationNormalizer.QR, seed=None, precision="mixed",
                 autotune=True, use_graph=True):
        a = as_smat(matrix)
        norm = power_iteration_normalizer
        if isinstance(norm, PowerIterationNormalizer):
            norm = norm.value
        offs = np.zeros(len(subsets) + 1, dtype=np.uint64)
        offs[1:] = np.cumsum([len(c) for c in subsets])
        cols = (np.concatenate([np.asarray(c, dtype=np.int64) for c in subsets]) if len(subsets)
                else np.zeros(0, np.int64))
        if cols.size and cols.min() < 0:
            raise ShapeError("Column index out of bounds", 6)
        cols = cols.astype(np.uint64)
        o = _abi.svdb_batch_options()
        _abi.lib().svdb_batch_options_default(C.byref(o))
        o.precision = _abi.PRECISION[precision]
        o.autotune = int(autotune)
        o.use_graph = int(use_graph)
        h = C.c_void_p()
        check(_abi.lib().svdb_batch_create(a.handle, offs.ctypes.data, cols.ctypes.data, len(subsets), target_rank,
                                           n_oversamples, n_power_iters, _abi.NORMALIZER[norm],
                                           int(seed is not None), 0 if seed is None else int(seed), C.byref(o),
                                           C.byref(h)))
        self._h = h
        self._matrix = a  # the batch reads the matrix's device arrays
        self.count = len(subsets)

    def run(self, results=True):
        """Replay the batch; results=False leaves the results on the device (timing)."""
        if not results:
            check(_abi.lib().svdb_batch_run(self._h, None))
            return None
        recs = (_abi.svdb_rec * self.count)()
        try:
            check(_abi.lib().svdb_batch_run(self._h, recs))
            return [rec_from_c(recs[i]) for i in range(self.count)]
        finally:
            for i in range(self.count):
                _abi.lib().svdb_rec_free(C.byref(recs[i]))

    def info(self) -> dict:
        inf = _abi.svdb_batch_info()
        check(_abi.lib().svdb_batch_get_info(self._h, C.byref(inf)))
        return {k: getattr(inf, k) for k, _ in inf._fields_}

    def close(self):
        if self._h:
            _abi.lib().svdb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def randomized_svd_batch(matrix, subsets, target_rank, n_oversamples, n_power_iters,
                         power_iteration_normalizer=PowerIterationNormalizer.QR, seed=None, precision="mixed"):
    """One-shot batch: prepare, run once, release."""
    b = RandomizedBatch(matrix, subsets, target_rank, n_oversamples, n_power_iters, power_iteration_normalizer,
                        seed, precision)
    try:
        return b.run()
    finally:
        b.close()
