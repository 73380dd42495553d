"""ecgpu — host side of the B200 closed-shell coupled-cluster library."""
from ._lib import ECGError, ECG_PREC_FP64, ECG_PREC_MIXED, lib, library_path  # noqa: F401
from .context import Context, Diis  # noqa: F401
