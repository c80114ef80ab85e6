"""B200 implementation of CUDA-CVDV's dense state-vector path.

``CudaCvdv`` and ``SeparableState`` mirror the reference's Python API; the work
runs in ``lib/libcvdv.so`` (hand-written sm_100a kernels behind a C ABI).
"""

from .cudaCvdv import CudaCvdv, CvdvError  # noqa: F401
from .separable import SeparableState  # noqa: F401
from . import _lib  # noqa: F401

__all__ = ["CudaCvdv", "CvdvError", "SeparableState"]
