"""lanczos::* (src/lanczos/mod.rs:27-189): LAS2 on the GPU, as the crate writes it."""
from __future__ import annotations

import ctypes as C

import numpy as np

from .. import _abi
from .._core import SvdRec, as_smat, check, options, rec_from_c
from .masked import MaskedCSRMatrix  # noqa: F401  (lanczos::masked)


def _run(fn, a, *args, opts=None, f32=False):
    r = _abi.svdb_rec_f32() if f32 else _abi.svdb_rec()
    try:
        check(fn(a.handle, *args, C.byref(opts) if opts is not None else None, C.byref(r)))
        return rec_from_c(r)
    finally:
        (_abi.lib().svdb_rec_f32_free if f32 else _abi.lib().svdb_rec_free)(C.byref(r))


def _las2_fn(a, algorithm):
    """(entry point, end_interval array type, T = f32?) for the matrix's scalar T."""
    if a.dtype == np.float32:
        return _abi.lib().svdb_las2_f32, C.c_float * 2, True
    fn = _abi.lib().svdb_legacy_svd_las2 if algorithm == "legacy" else _abi.lib().svdb_las2
    return fn, C.c_double * 2, False


def svd_las2(a, dimensions=0, iterations=0, end_interval=(-1.0e-30, 1.0e-30), kappa=1.0e-6, random_seed=0,
             precision="f64") -> SvdRec:
    """lanczos::svd_las2 (mod.rs:104-189), at the matrix's T (f64, or f32 for
    float32 matrices: f32 tolerances, float32 results; precision is ignored)."""
    a = as_smat(a)
    fn, eit, f32 = _las2_fn(a, "lanczos")
    return _run(fn, a, dimensions, iterations, eit(*end_interval), kappa, random_seed,
                opts=options(precision=precision, algorithm="lanczos"), f32=f32)


def svd(a) -> SvdRec:
    """lanczos::svd (mod.rs:27-36): svd_las2(A, 0, 0, [-1e-30, 1e-30], 1e-6, 0)."""
    return svd_las2(a, 0, 0, (-1.0e-30, 1.0e-30), 1.0e-6, 0)


def svd_dim(a, dimensions) -> SvdRec:
    """lanczos::svd_dim (mod.rs:45-55)."""
    return svd_las2(a, dimensions, 0, (-1.0e-30, 1.0e-30), 1.0e-6, 0)


def svd_dim_seed(a, dimensions, random_seed) -> SvdRec:
    """lanczos::svd_dim_seed (mod.rs:65-86)."""
    return svd_las2(a, dimensions, 0, (-1.0e-30, 1.0e-30), 1.0e-6, random_seed)


def las2_plan(nrows, ncols, nnz, dimensions=0, iterations=0):
    """Host-side argument handling of svd_las2 (mod.rs:116-145): (dimensions, iterations,
    transposed, sparsity branch 0..3).  Raises Las2Error for dimensions < 2."""
    d, it = C.c_uint64(), C.c_uint64()
    tr, br = C.c_int32(), C.c_int32()
    check(_abi.lib().svdb_las2_plan(nrows, ncols, nnz, dimensions, iterations, C.byref(d), C.byref(it),
                                    C.byref(tr), C.byref(br)))
    return int(d.value), int(it.value), bool(tr.value), int(br.value)


def start_vector(seed: int, n: int) -> np.ndarray:
    """The start vector startv draws on the device (mod.rs:598-605)."""
    out = np.zeros(n)
    check(_abi.lib().svdb_start_vector(seed, out.ctypes.data, n))
    return out


def las2_traced(a, dimensions=0, iterations=0, end_interval=(-1.0e-30, 1.0e-30), kappa=1.0e-6, random_seed=0,
                algorithm="lanczos", precision="f64"):
    """Run LAS2 and return its internals with the result:
    {"rec": SvdRec or None, "error": SvdLibError or None, "alf", "bet", "ritz", "bnd", "steps",
     "purges", "sparsity_branch", "lanczos_blocks"}."""
    a = as_smat(a)
    cap = min(a.nrows(), a.ncols()) + 4
    bufs = {k: np.zeros(cap) for k in ("alf", "bet", "ritz", "bnd")}
    tr = _abi.svdb_trace()
    for k, v in bufs.items():
        setattr(tr, k, v.ctypes.data_as(C.POINTER(C.c_double)))
    tr.cap = cap
    o = options(precision=precision, algorithm=algorithm)
    o.trace = C.pointer(tr)
    fn, eit, f32 = _las2_fn(a, algorithm)
    out = {"rec": None, "error": None}
    try:
        out["rec"] = _run(fn, a, dimensions, iterations, eit(*end_interval), kappa, random_seed, opts=o, f32=f32)
    except Exception as e:  # noqa: BLE001 - returned to the caller with the trace
        out["error"] = e
    st = int(tr.steps)
    out.update({"alf": bufs["alf"][: st + 1].copy(), "bet": bufs["bet"][: st + 2].copy(),
                "ritz": bufs["ritz"][: st + 1].copy(), "bnd": bufs["bnd"][: st + 1].copy(), "steps": st,
                "purges": int(tr.purges), "sparsity_branch": int(tr.sparsity_branch),
                "lanczos_blocks": int(tr.lanczos_blocks)})
    return out
