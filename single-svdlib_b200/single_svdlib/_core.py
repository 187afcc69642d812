"""Python mirror of single-svdlib's public types over the C ABI.

Names follow the crate: ``SvdRec`` / ``Diagnostics`` (src/utils.rs:44-79),
``SvdLibError`` and its variants (src/error.rs:4-21), and the sparse matrix
types the crate accepts (nalgebra_sparse CsrMatrix / CscMatrix / CooMatrix,
src/lanczos/mod.rs:1415-1740).  Matrices are uploaded to the GPU when they are
constructed and keep a device handle for their lifetime.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi


# ----------------------------------------------------------------- errors --
class SvdLibError(Exception):
    """SvdLibError (src/error.rs:4-21); `kind` is the variant name."""

    kind = "SvdLibError"

    def __init__(self, msg: str, status: int):
        super().__init__(msg)
        self.status = status


class ImtqlbError(SvdLibError):
    kind = "ImtqlbError"


class StartvError(SvdLibError):
    kind = "StartvError"


class StponeError(SvdLibError):
    kind = "StponeError"


class Imtql2Error(SvdLibError):
    kind = "Imtql2Error"


class Las2Error(SvdLibError):
    kind = "Las2Error"


class ShapeError(SvdLibError):
    """Where the crate panics (assert!, ndarray shape mismatch)."""

    kind = "ShapeError"


class DeviceError(SvdLibError):
    """CUDA failure, device allocation failure or a device-side wait limit."""

    kind = "DeviceError"


class UnsupportedError(SvdLibError):
    kind = "Unsupported"


class NoConvergenceError(SvdLibError):
    """An iterative solve (the adjoint's block CG) stopped above its tolerance."""

    kind = "NoConvergence"


_ERR = {1: ImtqlbError, 2: StartvError, 3: StponeError, 4: Imtql2Error, 5: Las2Error, 6: ShapeError,
        7: DeviceError, 8: DeviceError, 9: UnsupportedError, 10: ValueError, 11: DeviceError,
        12: NoConvergenceError}


def check(status: int):
    if status == _abi.SVDB_OK:
        return
    cls = _ERR.get(status, SvdLibError)
    msg = _abi.last_error()
    if cls is ValueError:
        raise ValueError(msg)
    raise cls(msg, status)


# -------------------------------------------------------------- results ----
@dataclass
class Diagnostics:
    """Diagnostics<T> (src/utils.rs:67-79)."""

    non_zero: int
    dimensions: int
    iterations: int
    transposed: bool
    lanczos_steps: int
    ritz_values_stabilized: int
    significant_values: int
    singular_values: int
    end_interval: tuple
    kappa: float
    random_seed: int


@dataclass
class SvdRec:
    """SvdRec<T> (src/utils.rs:44-50).

    ``u`` keeps the crate's orientation: d x m from LAS2, m x d from
    randomized_svd.  ``times_ms`` holds the device phase timers of the call.
    """

    d: int
    u: np.ndarray
    s: np.ndarray
    vt: np.ndarray
    diagnostics: Diagnostics
    origin: int = 0
    times_ms: dict = field(default_factory=dict)

    @property
    def ut(self):  # legacy::SvdRec field name (src/legacy.rs:463)
        return self.u

    def recompose(self) -> np.ndarray:
        """SvdRec::recompose: u . diag(s) . vt as written (src/lanczos/mod.rs:1408-1413),
        ut^T . diag(s) . vt for legacy records (src/legacy.rs:2023-2028)."""
        if self.origin == _abi.ORIGIN_LEGACY:
            return (self.u.T * self.s) @ self.vt
        if self.u.shape[1] != self.d:
            raise ShapeError(f"ndarray: inputs {self.u.shape[0]} x {self.u.shape[1]} and {self.d} x {self.d} "
                             "are not compatible for matrix multiplication", 6)
        return (self.u * self.s) @ self.vt


def rec_from_c(r) -> SvdRec:
    """SvdRec from an svdb_rec (T = f64) or an svdb_rec_f32 (T = f32, float32 arrays)."""
    d = int(r.d)
    ur, uc, vr, vc = int(r.u_rows), int(r.u_cols), int(r.vt_rows), int(r.vt_cols)
    dtype = np.float32 if isinstance(r, _abi.svdb_rec_f32) else np.float64

    def arr(ptr, count, shape):
        if count == 0:
            return np.zeros(shape, dtype=dtype)
        return np.ctypeslib.as_array(ptr, (count,)).copy().reshape(shape)

    u = arr(r.u, ur * uc, (ur, uc))
    s = arr(r.s, d, (d,))
    vt = arr(r.vt, vr * vc, (vr, vc))
    dg = r.diagnostics
    diag = Diagnostics(int(dg.non_zero), int(dg.dimensions), int(dg.iterations), bool(dg.transposed),
                       int(dg.lanczos_steps), int(dg.ritz_values_stabilized), int(dg.significant_values),
                       int(dg.singular_values), (dg.end_interval[0], dg.end_interval[1]), float(dg.kappa),
                       int(dg.random_seed))
    times = {"total": r.time_ms_total, "spmv": r.time_ms_spmv, "ortho": r.time_ms_ortho,
             "tridiag": r.time_ms_tridiag, "ritvec": r.time_ms_ritvec}
    return SvdRec(d, u, s, vt, diag, int(r.origin), times)


def options(precision="f64", algorithm="lanczos", result_on_device=False, verbose=False, omega=None):
    o = _abi.svdb_options()
    _abi.lib().svdb_options_default(C.byref(o))
    o.precision = _abi.PRECISION[precision]
    o.algorithm = _abi.ALGORITHM[algorithm]
    o.result_on_device = int(result_on_device)
    o.verbose = int(verbose)
    if omega is not None:
        o.omega = omega.ctypes.data_as(C.POINTER(C.c_double))
    return o


# -------------------------------------------------------------- matrices ---
def _u64(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _values(data, kind):
    """(values, T, constructor): float32 values make a T = f32 matrix, anything
    else is taken as f64."""
    data = np.asarray(data)
    if data.dtype == np.float32:
        return np.ascontiguousarray(data), np.float32, getattr(_abi.lib(), f"svdb_matrix_create_{kind}_f32")
    return _f64(data), np.float64, getattr(_abi.lib(), f"svdb_matrix_create_{kind}")


class _Handle:
    """Owns an svdb_matrix handle (the SMat trait object).  ``dtype`` is the
    crate's scalar T of the matrix: float64, or float32 for matrices built
    from float32 values (the solvers then run at T = f32)."""

    _h = None
    dtype = np.float64

    def _take(self, h):
        self._h = h

    @property
    def handle(self):
        return self._h

    def nrows(self) -> int:
        return int(_abi.lib().svdb_matrix_nrows(self._h))

    def ncols(self) -> int:
        return int(_abi.lib().svdb_matrix_ncols(self._h))

    def nnz(self) -> int:
        return int(_abi.lib().svdb_matrix_nnz(self._h))

    @property
    def shape(self):
        return (self.nrows(), self.ncols())

    def close(self):
        if self._h:
            _abi.lib().svdb_matrix_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # SMat::svd_opa (src/utils.rs:26) and svd_opb (src/lanczos/mod.rs:311-319)
    def svd_opa(self, x, transposed=False) -> np.ndarray:
        x = _f64(x)
        y = np.zeros(self.ncols() if transposed else self.nrows())
        check(_abi.lib().svdb_opa(self._h, x.ctypes.data, y.ctypes.data, int(transposed)))
        return y

    def svd_opb(self, x, transposed=False) -> np.ndarray:
        x = _f64(x)
        y = np.zeros(self.nrows() if transposed else self.ncols())
        check(_abi.lib().svdb_opb(self._h, x.ctypes.data, y.ctypes.data, int(transposed)))
        return y

    # SMat::multiply_with_dense / multiply_transposed_by_dense (masked.rs:265-733), row-major
    def multiply_with_dense(self, dense, transpose_self=False) -> np.ndarray:
        dense = _f64(dense)
        l = dense.shape[1]
        out = np.zeros((self.ncols() if transpose_self else self.nrows(), l))
        check(_abi.lib().svdb_multiply_with_dense(self._h, dense.ctypes.data, l, out.ctypes.data,
                                                  int(transpose_self)))
        return out

    def multiply_transposed_by_dense(self, q) -> np.ndarray:
        q = _f64(q)
        l = q.shape[1]
        out = np.zeros((l, self.ncols()))
        check(_abi.lib().svdb_multiply_transposed_by_dense(self._h, q.ctypes.data, l, out.ctypes.data))
        return out

    # compute_column_means (masked.rs:240-263)
    def column_means(self) -> np.ndarray:
        out = np.zeros(self.ncols())
        check(_abi.lib().svdb_column_means(self._h, out.ctypes.data))
        return out

    # SMat::multiply_with_dense_centered / multiply_transposed_by_dense_centered
    # (src/utils.rs:29-32): exact products of A - 1 means^T
    def _means(self, means):
        means = _f64(means)
        if means.shape != (self.ncols(),):
            raise ShapeError(f"means has {means.size} values for {self.ncols()} columns")
        return means

    def multiply_with_dense_centered(self, dense, means, transpose_self=False) -> np.ndarray:
        dense, means = _f64(dense), self._means(means)
        if dense.shape[0] != (self.nrows() if transpose_self else self.ncols()):
            raise ShapeError("dense operand has the wrong number of rows")
        l = dense.shape[1]
        out = np.zeros((self.ncols() if transpose_self else self.nrows(), l))
        check(_abi.lib().svdb_multiply_with_dense_centered(self._h, dense.ctypes.data, l, means.ctypes.data,
                                                           out.ctypes.data, int(transpose_self)))
        return out

    def multiply_transposed_by_dense_centered(self, q, means) -> np.ndarray:
        q, means = _f64(q), self._means(means)
        if q.shape[0] != self.nrows():
            raise ShapeError("q has the wrong number of rows")
        l = q.shape[1]
        out = np.zeros((l, self.ncols()))
        check(_abi.lib().svdb_multiply_transposed_by_dense_centered(self._h, q.ctypes.data, l, means.ctypes.data,
                                                                    out.ctypes.data))
        return out


class CsrMatrix(_Handle):
    """nalgebra_sparse::CsrMatrix<f64>, uploaded to the current CUDA device."""

    def __init__(self, nrows, ncols, indptr, indices, data):
        indptr, indices = _u64(indptr), _u64(indices)
        data, self.dtype, fn = _values(data, "csr")
        h = C.c_void_p()
        check(fn(nrows, ncols, len(data), indptr.ctypes.data, indices.ctypes.data, data.ctypes.data, C.byref(h)))
        self._take(h)

    @classmethod
    def from_scipy(cls, m):
        m = m.tocsr()
        return cls(m.shape[0], m.shape[1], m.indptr, m.indices, m.data)


class CscMatrix(_Handle):
    """nalgebra_sparse::CscMatrix<f64>."""

    def __init__(self, nrows, ncols, indptr, indices, data):
        indptr, indices = _u64(indptr), _u64(indices)
        data, self.dtype, fn = _values(data, "csc")
        h = C.c_void_p()
        check(fn(nrows, ncols, len(data), indptr.ctypes.data, indices.ctypes.data, data.ctypes.data, C.byref(h)))
        self._take(h)

    @classmethod
    def from_scipy(cls, m):
        m = m.tocsc()
        return cls(m.shape[0], m.shape[1], m.indptr, m.indices, m.data)


class CooMatrix(_Handle):
    """nalgebra_sparse::CooMatrix<f64>: triplets in push order, duplicates kept."""

    def __init__(self, nrows, ncols, rows, cols, data):
        rows, cols = _u64(rows), _u64(cols)
        data, self.dtype, fn = _values(data, "coo")
        h = C.c_void_p()
        check(fn(nrows, ncols, len(data), rows.ctypes.data, cols.ctypes.data, data.ctypes.data, C.byref(h)))
        self._take(h)


class MaskedCSRMatrix(_Handle):
    """MaskedCSRMatrix (src/lanczos/masked.rs:13-66): a column subset of a CsrMatrix.

    The parent must outlive the view (the crate's borrow); the view keeps a
    reference to it.
    """

    def __init__(self, matrix: CsrMatrix, column_mask):
        mask = np.ascontiguousarray(column_mask, dtype=np.uint8)
        h = C.c_void_p()
        check(_abi.lib().svdb_masked_new(matrix.handle, mask.ctypes.data, len(mask), C.byref(h)))
        self._parent = matrix
        self.dtype = matrix.dtype
        self._take(h)

    @classmethod
    def new(cls, matrix, column_mask):
        return cls(matrix, column_mask)

    @classmethod
    def with_columns(cls, matrix: CsrMatrix, columns):
        cols = _u64(columns)
        obj = cls.__new__(cls)
        h = C.c_void_p()
        check(_abi.lib().svdb_masked_with_columns(matrix.handle, cols.ctypes.data, len(cols), C.byref(h)))
        obj._parent = matrix
        obj.dtype = matrix.dtype
        obj._take(h)
        return obj

    def uses_all_columns(self) -> bool:
        return _abi.lib().svdb_masked_uses_all_columns(self._h) == 1

    def maps(self):
        """(masked_to_original, original_to_masked with -1 for None)."""
        m2o = np.zeros(max(self.ncols(), 1), dtype=np.int64)
        o2m = np.zeros(max(self._parent.ncols(), 1), dtype=np.int64)
        check(_abi.lib().svdb_masked_maps(self._h, m2o.ctypes.data, o2m.ctypes.data))
        return m2o[: self.ncols()], o2m[: self._parent.ncols()]


class BorrowedMatrix(_Handle):
    """A matrix handle created through the C ABI directly (svdb_matrix_create_*);
    the caller keeps ownership and destroys it."""

    def __init__(self, handle):
        self._take(handle)

    def close(self):
        self._h = None


def as_smat(a):
    """Accept the package's matrix types or a scipy.sparse matrix (uploaded as CSR)."""
    if isinstance(a, _Handle):
        return a
    if hasattr(a, "tocsr"):
        return CsrMatrix.from_scipy(a)
    raise TypeError(f"not a sparse matrix: {type(a)!r}")
