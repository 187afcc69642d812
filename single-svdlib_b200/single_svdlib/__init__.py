"""single_svdlib on B200: the hot path of single-svdlib 1.0.9 as CUDA kernels for sm_100a.

Mirrors the crate's public API (src/lib.rs:1-9): ``lanczos`` (svd, svd_dim,
svd_dim_seed, svd_las2, masked.MaskedCSRMatrix), ``randomized``
(randomized_svd, PowerIterationNormalizer), ``legacy`` (SVDLIBC semantics),
``SvdRec`` / ``Diagnostics`` and the ``SvdLibError`` variants.  All work runs
in libsvdb200.so through its C ABI (include/svdb200.h).
"""
from . import lanczos, legacy, randomized  # noqa: F401
from ._abi import LIB_PATH  # noqa: F401
from ._core import (CooMatrix, CscMatrix, CsrMatrix, DeviceError, Diagnostics, Imtql2Error,  # noqa: F401
                    ImtqlbError, Las2Error, MaskedCSRMatrix, ShapeError, StartvError, StponeError, SvdLibError,
                    SvdRec, UnsupportedError)
