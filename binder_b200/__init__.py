"""binder_b200: B200-native (sm_100a) engine for BINDER's registration + Gibbs-sampling hot path.

``binder_b200._core`` mirrors the reference's ``BINDER._core`` extension (Registration,
NonLinearTransformation, topology_correction_3D, compute_jacobian_determinant_3D) over the C ABI
declared in include/binder_b200.h.  ``binder_b200.utils`` holds the host-side helpers the
reference's Python layer feeds the engine with (D matrix, robust binning).
"""
from ._lib import LIB_PATH, BinderError  # noqa: F401

__all__ = ["LIB_PATH", "BinderError"]
