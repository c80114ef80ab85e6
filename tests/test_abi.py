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
