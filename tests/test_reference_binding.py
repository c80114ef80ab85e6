"""The reference's own, unmodified Python binding loads this library.

The reference's ``CudaCvdv`` (src/cudaCvdv.py:17-74) finds ``libcvdv.so`` through
its module global ``build_dir`` and declares argtypes/restypes for every symbol
it calls.  Pointing ``build_dir`` at this library's directory is the whole
drop-in step; this test does exactly that with the stock module and checks
that every binding the stock loader makes resolves to this library's export.

No CUDA call is made (the stock loader only opens the library and declares
signatures), so the test runs on CPU.  It needs a checkout of the reference:
``CVDV_REFERENCE=/path/to/reference``, or a ``reference`` directory beside this
repository; without one it is skipped.
"""

import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "cuda-cvdv_b200", "lib")


def _reference_dir():
    for cand in (os.environ.get("CVDV_REFERENCE"), os.path.join(os.path.dirname(ROOT), "reference")):
        if cand and os.path.isfile(os.path.join(cand, "src", "cudaCvdv.py")):
            return cand
    return None


@pytest.fixture(scope="module")
def stock_module():
    ref = _reference_dir()
    if ref is None:
        pytest.skip("no reference checkout (set CVDV_REFERENCE)")
    if not os.path.exists(os.path.join(LIBDIR, "libcvdv.so")):
        pytest.skip("libcvdv.so not built")
    saved = {k: v for k, v in sys.modules.items() if k == "src" or k.startswith("src.")}
    for k in saved:
        del sys.modules[k]
    sys.path.insert(0, ref)
    try:
        mod = importlib.import_module("src.cudaCvdv")
        yield mod
    finally:
        sys.path.remove(ref)
        for k in [k for k in sys.modules if k == "src" or k.startswith("src.")]:
            del sys.modules[k]
        sys.modules.update(saved)


def test_stock_loader_binds_every_symbol(stock_module):
    import ctypes
    stock_module.build_dir = LIBDIR  # the one change a user makes
    stock_module._lib = None
    lib = stock_module._get_lib()
    assert os.path.samefile(lib._name, os.path.join(LIBDIR, "libcvdv.so"))
    # every function the stock loader declared is this library's symbol
    ours = ctypes.CDLL(os.path.join(LIBDIR, "libcvdv.so"))
    declared = [n for n in dir(lib) if n.startswith("cvdv")]
    assert len(declared) >= 30
    for name in declared:
        assert hasattr(ours, name), name
    # the return types the stock class relies on
    assert lib.cvdvCreate.restype is ctypes.c_void_p
    assert lib.cvdvGetNorm.restype is ctypes.c_double
    assert lib.cvdvGetPhotonNumber.restype is ctypes.c_double
    # and the class the stock module exports is the one that drives it
    assert hasattr(stock_module.CudaCvdv, "getWigner")
