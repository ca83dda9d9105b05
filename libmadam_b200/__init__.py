"""libmadam_b200: the Madam destriping solve on NVIDIA B200 (sm_100a).

The compute path is the in-tree CUDA library libmadam.so; there is no CPU
fallback.  `libmadam_b200.libmadam_wrapper` is the drop-in for the
reference's `libmadam_wrapper` module.
"""
from ._lib import build, load, last_error, LIB_PATH  # noqa: F401

__all__ = ["build", "load", "last_error", "LIB_PATH"]
