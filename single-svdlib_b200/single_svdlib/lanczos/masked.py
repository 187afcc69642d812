"""lanczos::masked (src/lanczos/masked.rs)."""
from .._core import MaskedCSRMatrix  # noqa: F401
