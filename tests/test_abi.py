"""CPU checks of the boundary: the library loads, exports every symbol declared
in include/cvdv.h, and the Python binding declares each of them.  No call here
touches the GPU."""

import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "cvdv.h")
LIB = os.path.join(ROOT, "cuda-cvdv_b200", "lib", "libcvdv.so")

# the reference's extern "C" set (src/cuda/api.h:14-61) and the names its
# Python wrapper binds (src/cudaCvdv.py:34-73)
REFERENCE_API = """cvdvCreate cvdvDestroy cvdvFree cvdvInitFromSeparable cvdvSetStateFromDevicePtr
cvdvGetNumRegisters cvdvGetTotalSize cvdvGetRegisterInfo cvdvGetRegisterDim cvdvGetRegisterDx
cvdvFtQ2P cvdvFtP2Q cvdvDisplacement cvdvConditionalDisplacement cvdvPauliRotation cvdvHadamard
cvdvParity cvdvConditionalParity cvdvSwapRegisters cvdvPhaseSquare cvdvPhaseCubic cvdvRotation
cvdvConditionalRotation cvdvSqueeze cvdvConditionalSqueeze cvdvBeamSplitter
cvdvConditionalBeamSplitter cvdvQ1Q2Gate cvdvGetWigner cvdvGetHusimiQ cvdvGetHusimiQOverlap
cvdvGetHusimiQWigner cvdvMeasureMultiple cvdvMeasureMultipleCT cvdvGetState cvdvGetNorm
cvdvGetFidelity cvdvGetPhotonNumber cvdvFidelityStatevectors""".split()


def header_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(cvdv[A-Za-z0-9]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib_path():
    if not os.path.exists(LIB):
        import sys
        sys.path.insert(0, ROOT)
        import __graft_entry__ as g
        g.build()
    assert os.path.exists(LIB)
    return LIB


def test_header_covers_reference_api():
    syms = set(header_symbols())
    missing = [s for s in REFERENCE_API if s not in syms]
    assert not missing, missing


def test_library_exports_every_header_symbol(lib_path):
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (cvdv\w+)", out))
    missing = [s for s in header_symbols() if s not in exported]
    assert not missing, missing


def test_library_loads_and_binding_declares_all(lib_path):
    lib = ctypes.CDLL(lib_path)
    for s in header_symbols():
        assert hasattr(lib, s), s
    from cvdv_b200 import _lib
    bound = {name for name, _, _ in _lib.SIGNATURES}
    assert set(header_symbols()) <= bound, set(header_symbols()) - bound


def test_no_forbidden_libraries(lib_path):
    out = subprocess.run(["ldd", lib_path], capture_output=True, text=True).stdout
    for bad in ("cufft", "cutensor", "cublas"):
        assert bad not in out, out


def test_no_cpu_fallback_in_product():
    """The product package never imports the oracle."""
    pkg = os.path.join(ROOT, "cuda-cvdv_b200", "cvdv_b200")
    for f in os.listdir(pkg):
        if f.endswith(".py"):
            assert "oracle" not in open(os.path.join(pkg, f)).read(), f


def test_batch_struct_layouts_match(lib_path):
    """The numpy record layouts the host builds match the C structs of the stage kernel."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "cuda-cvdv_b200"))
    from cvdv_b200 import batch
    sizes = batch.struct_sizes()
    assert sizes == (batch.PHASE_DTYPE.itemsize, batch.PROGRAM_DTYPE.itemsize, batch.TASK_DTYPE.itemsize)


def test_error_paths_without_device(lib_path):
    """The reference prints or throws through the C ABI; this library records an
    error code and message and leaves outputs untouched.  Only argument checks
    that come before any CUDA call are exercised here: invalid creation
    arguments, calls on an empty context, null pointers."""
    lib = ctypes.CDLL(lib_path)
    vp = ctypes.c_void_p
    lib.cvdvCreateEx.restype = vp
    lib.cvdvCreateEx.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int]
    lib.cvdvGetLastError.restype = ctypes.c_int
    lib.cvdvGetLastError.argtypes = [vp, ctypes.c_char_p, ctypes.c_int]
    lib.cvdvGetNumRegisters.argtypes = [vp]
    lib.cvdvGetTotalSize.restype = ctypes.c_size_t
    lib.cvdvGetTotalSize.argtypes = [vp]
    lib.cvdvGetNorm.restype = ctypes.c_double
    lib.cvdvGetNorm.argtypes = [vp]
    lib.cvdvDisplacement.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double]
    lib.cvdvInitFromSeparable.argtypes = [vp, ctypes.POINTER(vp), ctypes.c_int]
    lib.cvdvMeasureMultiple.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_double)]
    lib.cvdvClearError.argtypes = [vp]
    lib.cvdvDestroy.argtypes = [vp]
    lib.cvdvMeasureMultipleNoAlloc.restype = ctypes.c_int
    lib.cvdvMeasureMultipleNoAlloc.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                               ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                               ctypes.POINTER(ctypes.c_double), vp]

    def err(ctx):
        buf = ctypes.create_string_buffer(256)
        return lib.cvdvGetLastError(ctx, buf, 256), buf.value.decode()

    def ints(*v):
        return (ctypes.c_int * len(v))(*v)

    # empty context (context.cu:10-12 of the reference): no registers, no error
    empty = lib.cvdvCreateEx(0, None, 0)
    assert empty and err(empty)[0] == 0
    assert lib.cvdvGetNumRegisters(empty) == 0 and lib.cvdvGetTotalSize(empty) == 1
    # invalid creation arguments are recorded on the returned handle
    for n, q, prec in [(65, [1] * 65, 0), (2, [3, 40], 0), (2, [3, 0], 0), (1, [3], 7), (2, [20, 20], 0)]:
        ctx = lib.cvdvCreateEx(n, ints(*q), prec)
        code, msg = err(ctx)
        assert code == 1 and msg.startswith("cvdvCreate"), (n, q, prec, code, msg)
        lib.cvdvDestroy(ctx)
    # calls on a context without registers or state: error recorded, output untouched
    lib.cvdvDisplacement(empty, 0, 0.5, 0.0)
    assert err(empty)[0] != 0
    lib.cvdvClearError(empty)
    assert err(empty) == (0, "")
    lib.cvdvInitFromSeparable(empty, None, 0)
    assert err(empty)[0] == 2
    out = (ctypes.c_double * 2)(7.0, 7.0)
    lib.cvdvMeasureMultiple(empty, ints(0), 1, out)
    assert err(empty)[0] != 0 and list(out) == [7.0, 7.0]
    assert lib.cvdvGetNorm(empty) == 0.0 and err(empty)[0] == 2
    lib.cvdvDestroy(empty)
    # the allocation-free marginal rejects null pointers before touching the device
    assert lib.cvdvMeasureMultipleNoAlloc(None, 0, ints(1), 1, ints(0), 1, out, None) == 1
    assert list(out) == [7.0, 7.0]


def test_batch_row_task_shapes():
    """Row-task shapes the stage kernel takes: a row fits 512 threads, complex128 at
    most 16 amplitudes a thread; the defaults are among them."""
    from cvdv_b200.batch import default_loge, loge_options
    assert loge_options(8, 1) == [3, 4, 5] and loge_options(14, 1) == [5]
    assert loge_options(13, 1) == [4, 5] and loge_options(13, 0) == [4]
    assert loge_options(12, 0) == [3, 4]
    for prec, top in ((1, 14), (0, 13)):
        for m in range(8, top + 1):
            assert default_loge(m, prec) in loge_options(m, prec)
