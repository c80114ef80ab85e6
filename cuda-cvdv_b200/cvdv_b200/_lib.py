"""ctypes binding of libcvdv.so (the B200 build of the C ABI in include/cvdv.h).

The binding mirrors the reference's own loader (src/cudaCvdv.py:19-74): one
process-wide handle, argtypes declared once.  The library is loaded from the
package's ``lib/`` directory (or ``$CVDV_LIB``); if it is missing the import
fails loudly -- there is no CPU fallback.
"""

from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_size_t, c_void_p
from typing import Optional

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.environ.get("CVDV_LIB", os.path.join(PKG_DIR, "lib", "libcvdv.so"))

_lib: Optional[ctypes.CDLL] = None

# (name, argtypes, restype) for every exported entry point
SIGNATURES = [
    ("cvdvCreate", [c_int, POINTER(c_int)], c_void_p),
    ("cvdvCreateEx", [c_int, POINTER(c_int), c_int], c_void_p),
    ("cvdvDestroy", [c_void_p], None),
    ("cvdvFree", [c_void_p], None),
    ("cvdvInitFromSeparable", [c_void_p, POINTER(c_void_p), c_int], None),
    ("cvdvSetStateFromDevicePtr", [c_void_p, c_void_p], None),
    ("cvdvGetNumRegisters", [c_void_p], c_int),
    ("cvdvGetTotalSize", [c_void_p], c_size_t),
    ("cvdvGetRegisterInfo", [c_void_p, POINTER(c_int), POINTER(c_double)], None),
    ("cvdvGetRegisterDim", [c_void_p, c_int], c_int),
    ("cvdvGetRegisterDx", [c_void_p, c_int], c_double),
    ("cvdvFtQ2P", [c_void_p, c_int], None),
    ("cvdvFtP2Q", [c_void_p, c_int], None),
    ("cvdvDisplacement", [c_void_p, c_int, c_double, c_double], None),
    ("cvdvConditionalDisplacement", [c_void_p, c_int, c_int, c_int, c_double, c_double], None),
    ("cvdvPauliRotation", [c_void_p, c_int, c_int, c_int, c_double], None),
    ("cvdvHadamard", [c_void_p, c_int, c_int], None),
    ("cvdvParity", [c_void_p, c_int], None),
    ("cvdvConditionalParity", [c_void_p, c_int, c_int, c_int], None),
    ("cvdvSwapRegisters", [c_void_p, c_int, c_int], None),
    ("cvdvPhaseSquare", [c_void_p, c_int, c_double], None),
    ("cvdvPhaseCubic", [c_void_p, c_int, c_double], None),
    ("cvdvRotation", [c_void_p, c_int, c_double], None),
    ("cvdvConditionalRotation", [c_void_p, c_int, c_int, c_int, c_double], None),
    ("cvdvSqueeze", [c_void_p, c_int, c_double], None),
    ("cvdvConditionalSqueeze", [c_void_p, c_int, c_int, c_int, c_double], None),
    ("cvdvBeamSplitter", [c_void_p, c_int, c_int, c_double], None),
    ("cvdvConditionalBeamSplitter", [c_void_p, c_int, c_int, c_int, c_int, c_double], None),
    ("cvdvQ1Q2Gate", [c_void_p, c_int, c_int, c_double], None),
    ("cvdvGetWigner", [c_void_p, c_int, POINTER(c_double)], None),
    ("cvdvGetHusimiQ", [c_void_p, c_int, POINTER(c_double)], None),
    ("cvdvGetHusimiQOverlap", [c_void_p, c_int, POINTER(c_double)], None),
    ("cvdvGetHusimiQWigner", [c_void_p, c_int, POINTER(c_double)], None),
    ("cvdvMeasureMultiple", [c_void_p, POINTER(c_int), c_int, POINTER(c_double)], None),
    ("cvdvMeasureMultipleCT", [c_void_p, POINTER(c_int), c_int, POINTER(c_double)], None),
    ("cvdvGetState", [c_void_p, POINTER(c_double), POINTER(c_double)], None),
    ("cvdvGetNorm", [c_void_p], c_double),
    ("cvdvGetFidelity", [c_void_p, POINTER(c_void_p), c_int, POINTER(c_double)], None),
    ("cvdvGetPhotonNumber", [c_void_p, c_int], c_double),
    ("cvdvFidelityStatevectors", [c_void_p, c_void_p, POINTER(c_double)], None),
    ("cvdvGetPrecision", [c_void_p], c_int),
    ("cvdvGetLastError", [c_void_p, c_char_p, c_int], c_int),
    ("cvdvClearError", [c_void_p], None),
    ("cvdvSynchronize", [c_void_p], None),
    ("cvdvFlush", [c_void_p], None),
    ("cvdvPendingStages", [c_void_p], c_int),
    ("cvdvGetStateDevicePtr", [c_void_p], c_void_p),
    ("cvdvGetStream", [c_void_p], c_void_p),
    ("cvdvMeasureEach", [c_void_p, POINTER(c_int), c_int, POINTER(c_double)], None),
    ("cvdvSeparableFill", [c_void_p, c_int, c_int, POINTER(c_double), c_int, c_void_p], c_int),
    ("cvdvMeasureMultipleNoAlloc",
     [c_void_p, c_int, POINTER(c_int), c_int, POINTER(c_int), c_int, c_void_p, c_void_p], c_int),
    ("cvdvBatchRx", [c_void_p, c_int, c_int, c_int, c_int, c_void_p, c_double, c_void_p], c_int),
    ("cvdvBatchCondDisp", [c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_double, c_void_p], c_int),
    ("cvdvBatchRxAdjoint", [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p], c_int),
    ("cvdvBatchCondDispAdjoint",
     [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p], c_int),
    ("cvdvBatchRxCondDisp", [c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p], c_int),
    ("cvdvBatchRxCondDispAdjoint",
     [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p],
     c_int),
    ("cvdvBatchOverlap", [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_void_p, c_void_p], c_int),
    ("cvdvBatchStructSizes", [POINTER(c_int)], None),
    ("cvdvBatchRunStage", [c_void_p, c_int, c_void_p, c_int, c_void_p, c_int, c_void_p], c_int),
    ("cvdvLaunchCount", [], ctypes.c_ulonglong),
    ("cvdvSetFusion", [c_void_p, c_int], None),
    ("cvdvCancelledTransforms", [c_void_p], ctypes.c_longlong),
    ("cvdvSetTiming", [c_void_p, c_int], None),
    ("cvdvGetKernelStats", [c_void_p, POINTER(c_double), POINTER(ctypes.c_longlong), c_int], c_int),
]

KERNEL_KINDS = ["fft_pass", "pair", "diag", "perm", "table", "init", "reduce", "phase_space", "seq", "col", "col_tc"]


def kernel_stats(ctx):
    """Per-kind (ms, launches) since the last call, when timing is on."""
    n = len(KERNEL_KINDS)
    ms = (c_double * n)()
    cnt = (ctypes.c_longlong * n)()
    load().cvdvGetKernelStats(ctx, ms, cnt, n)
    return {k: (ms[i], int(cnt[i])) for i, k in enumerate(KERNEL_KINDS)}


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libcvdv.so and declare every signature (no CUDA call is made)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"libcvdv.so not found at {path}; build it with `python -c 'import __graft_entry__ as g; g.build()'`"
            " or `make -C cuda-cvdv_b200/csrc`")
    lib = ctypes.CDLL(path)
    for name, args, res in SIGNATURES:
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def last_error(ctx=None) -> tuple[int, str]:
    buf = ctypes.create_string_buffer(512)
    code = load().cvdvGetLastError(ctx, buf, 512)
    return int(code), buf.value.decode(errors="replace")
