"""legacy::* (src/legacy.rs:438-654): LAS2 with SVDLIBC semantics, on the GPU."""
from __future__ import annotations

import ctypes as C

from . import _abi
from ._core import SvdRec, as_smat, options
from .lanczos import _run


def svdLAS2(a, dimensions=0, iterations=0, end_interval=(-1.0e-30, 1.0e-30), kappa=1.0e-6, random_seed=0,
            precision="f64") -> SvdRec:  # noqa: N802 (crate name)
    """legacy::svdLAS2 (legacy.rs:569-654)."""
    a = as_smat(a)
    ei = (C.c_double * 2)(*end_interval)
    return _run(_abi.lib().svdb_legacy_svd_las2, a, dimensions, iterations, ei, kappa, random_seed,
                opts=options(precision=precision, algorithm="legacy"))


svd_las2 = svdLAS2


def svd(a) -> SvdRec:
    """legacy::svd (legacy.rs:498-507)."""
    return svdLAS2(a, 0, 0, (-1.0e-30, 1.0e-30), 1.0e-6, 0)


def svd_dim(a, dimensions) -> SvdRec:
    """legacy::svd_dim (legacy.rs:516-525)."""
    return svdLAS2(a, dimensions, 0, (-1.0e-30, 1.0e-30), 1.0e-6, 0)


def svd_dim_seed(a, dimensions, random_seed) -> SvdRec:
    """legacy::svd_dim_seed (legacy.rs:535-550)."""
    return svdLAS2(a, dimensions, 0, (-1.0e-30, 1.0e-30), 1.0e-6, random_seed)
