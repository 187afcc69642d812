"""ctypes wrapper around the CPU checker (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY.  This module is the checker for the CUDA
implementation: only tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline / --impl reference legs may import it.  The product package never
imports it and has no CPU fallback.

Sparse inputs are numpy arrays; the dict returned by ``las2`` mirrors
``SvdRec`` plus the run's internals (alf, bet, ritz, bnd, steps) used by the
parity tests.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATHS = {"f64": os.path.join(_HERE, "_build", "liboracle.so"),
              "f32": os.path.join(_HERE, "_build", "liboracle_f32.so")}
_libs = {}

KIND = {"csr": 0, "csc": 1, "coo": 2, "masked": 3}
ERRORS = {0: "ok", 1: "ImtqlbError", 2: "StartvError", 3: "StponeError", 4: "Imtql2Error",
          5: "Las2Error", 6: "Shape", 9: "Unsupported", 10: "Panic"}


class OracleError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code
        self.kind = ERRORS.get(code, str(code))


class _Las2Out(C.Structure):
    _fields_ = [("d", C.c_uint64), ("ut_rows", C.c_uint64), ("ut_cols", C.c_uint64),
                ("vt_rows", C.c_uint64), ("vt_cols", C.c_uint64),
                ("ut", C.POINTER(C.c_double)), ("s", C.POINTER(C.c_double)), ("vt", C.POINTER(C.c_double)),
                ("dimensions", C.c_uint64), ("iterations", C.c_uint64), ("nnz", C.c_uint64),
                ("lanczos_steps", C.c_uint64), ("ritz_values_stabilized", C.c_uint64),
                ("significant_values", C.c_uint64), ("singular_values", C.c_uint64),
                ("transposed", C.c_int32), ("kappa", C.c_double), ("random_seed", C.c_uint32),
                ("steps", C.c_uint64), ("alf", C.POINTER(C.c_double)), ("bet", C.POINTER(C.c_double)),
                ("ritz", C.POINTER(C.c_double)), ("bnd", C.POINTER(C.c_double)),
                ("purges", C.c_uint64), ("sparsity", C.c_double), ("imtqlb_warned", C.c_int32),
                ("masked_would_panic", C.c_int32)]


class _RandOut(C.Structure):
    _fields_ = [("d", C.c_uint64), ("m", C.c_uint64), ("n", C.c_uint64),
                ("u", C.POINTER(C.c_double)), ("s", C.POINTER(C.c_double)), ("vt", C.POINTER(C.c_double)),
                ("t_sparse", C.c_double), ("t_rows", C.c_double), ("t_fixed", C.c_double)]


def build():
    """Compile the checker with its Makefile (g++, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib(scalar="f64"):
    """The checker built for the crate's scalar T: "f64" (every solver) or
    "f32" (lanczos and randomized; legacy is f64-only in the crate).  Arrays
    cross the interface as float64 either way."""
    if scalar not in _libs:
        path = _LIB_PATHS[scalar]
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        p = np.ctypeslib.ndpointer
        u64, f64, u8, i64 = (p(np.uint64, flags="C"), p(np.float64, flags="C"), p(np.uint8, flags="C"),
                             p(np.int64, flags="C"))
        L.orc_last_error.restype = C.c_char_p
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_chacha_block.argtypes = [p(np.uint8, flags="C"), C.c_uint64, C.c_uint64, C.c_int,
                                       p(np.uint32, flags="C")]
        L.orc_start_vector.argtypes = [C.c_uint32, f64, C.c_size_t]
        if scalar == "f64":
            L.orc_pythag.argtypes = [C.c_double, C.c_double, C.c_int]
            L.orc_pythag.restype = C.c_double
            L.orc_imtqlb.argtypes = [C.c_size_t, f64, f64, f64, C.c_int, C.c_size_t]
            L.orc_imtql2.argtypes = [C.c_size_t, f64, f64, f64, C.c_int, C.c_size_t]
        assert L.orc_real_bytes() == (8 if scalar == "f64" else 4)
        L.orc_las2.argtypes = [C.c_int, C.c_uint64, C.c_uint64, C.c_uint64, u64, u64, f64, C.c_void_p,
                               C.c_uint64, C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_uint32,
                               C.c_int, C.POINTER(_Las2Out)]
        L.orc_las2_free.argtypes = [C.POINTER(_Las2Out)]
        L.orc_opa.argtypes = [C.c_int, C.c_uint64, C.c_uint64, C.c_uint64, u64, u64, f64, C.c_void_p,
                              f64, f64, C.c_int, C.c_int]
        L.orc_masked_maps.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, u64, u64, u8, i64,
                                      C.POINTER(C.c_uint64), i64, C.POINTER(C.c_uint64)]
        L.orc_masked_dense.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, u64, u64, f64, u8, C.c_int,
                                       f64, C.c_uint64, f64, C.c_int]
        L.orc_randomized.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, u64, u64, f64, C.c_void_p,
                                     C.c_uint64, C.c_uint64, C.c_uint64, C.c_int, f64, C.c_int, C.c_int,
                                     C.POINTER(_RandOut)]
        L.orc_rand_free.argtypes = [C.POINTER(_RandOut)]
        _libs[scalar] = L
    return _libs[scalar]


def set_threads(t: int):
    lib().orc_set_threads(int(t))


def _u64(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def chacha_block(key: bytes, counter: int, stream: int, rounds: int) -> np.ndarray:
    out = np.zeros(16, dtype=np.uint32)
    k = np.frombuffer(bytes(key).ljust(32, b"\0"), dtype=np.uint8).copy()
    lib().orc_chacha_block(k, counter, stream, rounds, out)
    return out


def start_vector(seed: int, n: int, scalar="f64") -> np.ndarray:
    out = np.zeros(n, dtype=np.float64)
    lib(scalar).orc_start_vector(seed, out, n)
    return out


def pythag(a, b, legacy=False):
    return lib().orc_pythag(a, b, int(legacy))


def imtqlb(d, e, legacy=False, max_it=100):
    d, e = _f64(d).copy(), _f64(e).copy()
    bnd = np.zeros_like(d)
    rc = lib().orc_imtqlb(len(d), d, e, bnd, int(legacy), max_it)
    if rc:
        raise OracleError(rc, lib().orc_last_error().decode())
    return d, bnd


def imtql2(d, e, legacy=False, max_it=50):
    n = len(d)
    d, e = _f64(d).copy(), _f64(e).copy()
    z = np.eye(n).ravel().copy()
    rc = lib().orc_imtql2(n, d, e, z, int(legacy), max_it)
    if rc:
        raise OracleError(rc, lib().orc_last_error().decode())
    return d, z.reshape(n, n)


def _sparse_args(kind, A):
    """A: dict with nrows, ncols and (indptr, indices, data) [csr/csc/masked] or (row, col, data) [coo]."""
    if kind == "coo":
        return _u64(A["row"]), _u64(A["col"]), _f64(A["data"])
    return _u64(A["indptr"]), _u64(A["indices"]), _f64(A["data"])


def las2(kind, A, dimensions=0, iterations=0, end_interval=(-1e-30, 1e-30), kappa=1e-6, seed=0,
         legacy=False, mask=None, scalar="f64"):
    """Run lanczos::svd_las2 (legacy=False) or legacy::svdLAS2 (legacy=True),
    at T = f64 or, for lanczos, T = f32 (values rounded to f32 on entry)."""
    if legacy and scalar != "f64":
        raise ValueError("legacy::svdLAS2 is f64-only")
    L = lib(scalar)
    p, i, v = _sparse_args(kind, A)
    mk = None
    if kind == "masked":
        mk = np.ascontiguousarray(mask, dtype=np.uint8)
    out = _Las2Out()
    rc = L.orc_las2(KIND[kind], A["nrows"], A["ncols"], len(v), p, i, v,
                    mk.ctypes.data if mk is not None else None, dimensions, iterations,
                    float(end_interval[0]), float(end_interval[1]), kappa, seed, int(legacy), C.byref(out))
    if rc:
        err = OracleError(rc, L.orc_last_error().decode())
        err.steps, err.neig = out.steps, out.ritz_values_stabilized
        raise err
    try:
        d = out.d
        res = {
            "d": d,
            "ut": np.ctypeslib.as_array(out.ut, (max(1, d * out.ut_cols),))[: d * out.ut_cols].reshape(
                d, out.ut_cols).copy(),
            "s": np.ctypeslib.as_array(out.s, (max(1, d),))[:d].copy(),
            "vt": np.ctypeslib.as_array(out.vt, (max(1, d * out.vt_cols),))[: d * out.vt_cols].reshape(
                d, out.vt_cols).copy(),
            "diagnostics": {
                "non_zero": out.nnz, "dimensions": out.dimensions, "iterations": out.iterations,
                "transposed": bool(out.transposed), "lanczos_steps": out.lanczos_steps,
                "ritz_values_stabilized": out.ritz_values_stabilized,
                "significant_values": out.significant_values, "singular_values": out.singular_values,
                "end_interval": tuple(end_interval), "kappa": out.kappa, "random_seed": out.random_seed,
            },
            "steps": out.steps,
            "alf": np.ctypeslib.as_array(out.alf, (out.steps + 1,)).copy(),
            "bet": np.ctypeslib.as_array(out.bet, (out.steps + 2,)).copy(),
            "ritz": np.ctypeslib.as_array(out.ritz, (out.steps + 1,)).copy(),
            "bnd": np.ctypeslib.as_array(out.bnd, (out.steps + 1,)).copy(),
            "purges": out.purges,
            "sparsity": out.sparsity,
            "imtqlb_warned": bool(out.imtqlb_warned),
            "masked_would_panic": bool(out.masked_would_panic),
        }
    finally:
        L.orc_las2_free(C.byref(out))
    return res


def opa(kind, A, x, transposed=False, legacy=False, mask=None, scalar="f64"):
    p, i, v = _sparse_args(kind, A)
    m, n = A["nrows"], A["ncols"]
    if kind == "masked":
        ncol_eff = int(np.count_nonzero(mask))
    else:
        ncol_eff = n
    ylen = ncol_eff if transposed else m
    y = np.zeros(ylen)
    mk = np.ascontiguousarray(mask, dtype=np.uint8) if mask is not None else None
    L = lib(scalar)
    rc = L.orc_opa(KIND[kind], m, n, len(v), p, i, v, mk.ctypes.data if mk is not None else None,
                   _f64(x), y, int(transposed), int(legacy))
    if rc:
        raise OracleError(rc, L.orc_last_error().decode())
    return y


def masked_maps(A, mask):
    mask = np.ascontiguousarray(mask, dtype=np.uint8)
    n = A["ncols"]
    m2o = np.zeros(n, dtype=np.int64)
    o2m = np.zeros(n, dtype=np.int64)
    nm, mnnz = C.c_uint64(), C.c_uint64()
    lib().orc_masked_maps(A["nrows"], n, len(A["indices"]), _u64(A["indptr"]), _u64(A["indices"]), mask,
                          m2o, C.byref(nm), o2m, C.byref(mnnz))
    return m2o[: nm.value].copy(), o2m, mnnz.value


def masked_dense(A, mask, op, X, compat_d3=False):
    """op: 'AX' (X: nmasked x l), 'ATX' (X: m x l), 'XTA' (X: m x l)."""
    mask = np.ascontiguousarray(mask, dtype=np.uint8)
    X = _f64(X)
    l = X.shape[1]
    nm = int(np.count_nonzero(mask))
    shape = {"AX": (A["nrows"], l), "ATX": (nm, l), "XTA": (l, nm)}[op]
    R = np.zeros(shape)
    lib().orc_masked_dense(A["nrows"], A["ncols"], len(A["indices"]), _u64(A["indptr"]), _u64(A["indices"]),
                           _f64(A["data"]), mask, {"AX": 0, "ATX": 1, "XTA": 2}[op], X, l, R, int(compat_d3))
    return R


def randomized(A, target_rank, n_oversamples, n_power_iters, normalizer="QR", omega=None, mask=None,
               compat_d3=False, mean_center=False, scalar="f64"):
    """Randomized SVD on the masked view (all columns when mask is None); omega is n_masked x l row-major
    (float64 draws, rounded to T inside as T::from_f64 does)."""
    mk = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    out = _RandOut()
    L = lib(scalar)
    rc = L.orc_randomized(A["nrows"], A["ncols"], len(A["indices"]), _u64(A["indptr"]), _u64(A["indices"]),
                              _f64(A["data"]), mk.ctypes.data if mk is not None else None, target_rank,
                              n_oversamples, n_power_iters, {"QR": 0, "LU": 1, "None": 2}[normalizer],
                              _f64(omega), int(compat_d3), int(mean_center), C.byref(out))
    if rc:
        raise OracleError(rc, L.orc_last_error().decode())
    try:
        d, m, n = out.d, out.m, out.n
        res = {"d": d,
               "u": np.ctypeslib.as_array(out.u, (max(1, m * d),))[: m * d].reshape(m, d).copy(),
               "s": np.ctypeslib.as_array(out.s, (max(1, d),))[:d].copy(),
               "vt": np.ctypeslib.as_array(out.vt, (max(1, d * n),))[: d * n].reshape(d, n).copy(),
               "times": {"sparse": out.t_sparse, "rows": out.t_rows, "fixed": out.t_fixed}}
    finally:
        L.orc_rand_free(C.byref(out))
    return res


# --------------------------------------------------------- numpy checkers ----
def _splitmix64(x):
    """splitmix64 finaliser (Steele, Lea and Flood 2014) on uint64 arrays, wrapping."""
    with np.errstate(over="ignore"):
        x = x + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return x ^ (x >> np.uint64(31))


def omega_stream(seed, n, l):
    """The library's seeded Omega (n x l, row-major), restated in numpy so that
    the checker and the CUDA solve draw the same matrix from the same seed.

    Entry i: two uniforms from splitmix64 of (key + 2i, key + 2i + 1) with
    key = splitmix64(seed ^ 0x5DEECE66D), then Box-Muller.  The crate itself
    draws Omega with rand_distr's Normal (src/randomized/mod.rs:299-313), whose
    stream is not restated here.  Values agree with the device's to a few ulps
    (the device evaluates cos(pi * 2u) with cospi)."""
    key = _splitmix64(np.array([np.uint64(seed) ^ np.uint64(0x5DEECE66D)], dtype=np.uint64))[0]
    i = np.arange(n * l, dtype=np.uint64)
    with np.errstate(over="ignore"):
        a = _splitmix64(key + np.uint64(2) * i)
        b = _splitmix64(key + np.uint64(2) * i + np.uint64(1))
    u1 = ((a >> np.uint64(11)).astype(np.float64) + 0.5) * (1.0 / 9007199254740992.0)
    u2 = (b >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return (np.sqrt(-2.0 * np.log(u1)) * np.cos(np.pi * (2.0 * u2))).reshape(n, l)


def svd_flip(u=None, v=None, u_based_decision=True):
    """svd_flip (src/randomized/mod.rs:332-438), restated in numpy on copies.

    u-based: column j of u decides by its first entry of largest magnitude (a
    strict > scan from max_abs = 0, :357-365); negative -> column j of u and
    row j of v (j < min(v.rows, u.cols), :383-391) are negated.  v-based: row
    i of v decides (:405-413); column i of u follows (:429-435).
    """
    if u is None and v is None:
        raise OracleError(5, "Both u and v cannot be None")
    u = None if u is None else np.array(u, dtype=np.float64, copy=True)
    v = None if v is None else np.array(v, dtype=np.float64, copy=True)

    def first_max(vec):
        best, idx = 0.0, 0
        for i, x in enumerate(vec):
            if abs(x) > best:
                best, idx = abs(x), i
        return idx

    if u_based_decision:
        if u is None:
            raise OracleError(5, "u cannot be None when u_based_decision is true")
        signs = np.array([-1.0 if u[first_max(u[:, j]), j] < 0 else 1.0 for j in range(u.shape[1])])
        u *= signs[None, :]
        if v is not None:
            t = min(v.shape[0], len(signs))
            v[:t] *= signs[:t, None]
    else:
        if v is None:
            raise OracleError(5, "v cannot be None when u_based_decision is false")
        signs = np.array([-1.0 if v[i, first_max(v[i])] < 0 else 1.0 for i in range(v.shape[0])])
        v *= signs[:, None]
        if u is not None:
            t = min(u.shape[1], len(signs))
            u[:, :t] *= signs[None, :t]
    return u, v


def sddmm(A, left, right):
    """out[e] = left[row(e)] . right[col(e)] for the CSR entries of A (numpy)."""
    rows = np.repeat(np.arange(A["nrows"]), np.diff(A["indptr"]))
    return np.einsum("ij,ij->i", left[rows], right[A["indices"]])
