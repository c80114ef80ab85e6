"""cvdvMeasureMultipleNoAlloc (joint marginal with a fixed device scratch array,
no device allocation) against cvdvMeasureMultiple, both called through the C ABI.

Collected last so that it also runs after every other test has used the library
in the same process; it must pass alone in a fresh process too.
"""

import ctypes

import numpy as np
import pytest
import torch

from cvdv_b200 import _lib
from cvdv_b200.cudaCvdv import PRECISIONS, CudaCvdv

pytestmark = pytest.mark.gpu

QUBITS = [2, 6, 4, 8]  # 2^20 amplitudes: every one of the 148 partial-histogram blocks is used
MAX_BINS = 4096


def _ints(v):
    return (ctypes.c_int * len(v))(*v)


def _state(precision):
    rng = np.random.default_rng(11)
    n = 1 << sum(QUBITS)
    psi = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    psi /= np.linalg.norm(psi)
    sim = CudaCvdv(QUBITS, precision=precision)
    sim.initFromArray(psi)
    sim.cd(1, 0, 1, 0.7 + 0.2j)  # leave gates queued: the state pointer call flushes them
    sim.h(0, 0)
    return sim


def _existing(sim, regs):
    L = _lib.load()
    out = np.zeros(1 << sum(QUBITS[r] for r in regs), dtype=np.float64)
    L.cvdvMeasureMultiple(sim.ctx, _ints(regs), len(regs), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert _lib.last_error(sim.ctx)[0] == 0
    return out


def _no_alloc(sim, regs, bins, check_free=False):
    L = _lib.load()
    state = L.cvdvGetStateDevicePtr(sim.ctx)
    stream = L.cvdvGetStream(sim.ctx)
    out = torch.full((bins,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    code = L.cvdvMeasureMultipleNoAlloc(state, PRECISIONS[sim.precision], _ints(QUBITS), len(QUBITS),
                                        _ints(regs), len(regs), ctypes.c_void_p(out.data_ptr()), stream)
    L.cvdvSynchronize(sim.ctx)
    if check_free:
        assert torch.cuda.mem_get_info()[0] == free0, "device memory changed during the call"
    return code, out.cpu().numpy()


@pytest.mark.parametrize("precision", ["complex128", "complex64"])
def test_no_alloc_marginal_matches_existing(precision):
    sim = _state(precision)
    # first call: the largest marginal allowed (6 + 4 + 2 qubits = 4096 outcomes)
    regs = [1, 2, 0]
    code, got = _no_alloc(sim, regs, MAX_BINS)
    assert code == 0, _lib.last_error()
    ref = _existing(sim, regs)
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-15)
    # second call in a row: a smaller marginal reuses the scratch left by the first
    regs = [3]
    code, got = _no_alloc(sim, regs, 1 << QUBITS[3], check_free=True)
    assert code == 0, _lib.last_error()
    ref = _existing(sim, regs)
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-15)
    assert abs(got.sum() - 1.0) < 1e-6


_FIRST_CALL = r"""
import ctypes, sys
import numpy as np, torch
sys.path.insert(0, sys.argv[1])
from cvdv_b200 import _lib
from cvdv_b200.cudaCvdv import CudaCvdv
q = [2, 6, 4, 8]
rng = np.random.default_rng(3)
psi = rng.standard_normal(1 << 20) + 1j * rng.standard_normal(1 << 20)
sim = CudaCvdv(q)  # any context on the device loads the entry point's device code
sim.initFromArray(psi / np.linalg.norm(psi))
L = _lib.load()
ints = lambda v: (ctypes.c_int * len(v))(*v)
out = torch.zeros(256, dtype=torch.float64, device="cuda")
state = L.cvdvGetStateDevicePtr(sim.ctx)
torch.cuda.synchronize()
free0 = torch.cuda.mem_get_info()[0]
code = L.cvdvMeasureMultipleNoAlloc(state, 0, ints(q), 4, ints([3]), 1, ctypes.c_void_p(out.data_ptr()),
                                    L.cvdvGetStream(sim.ctx))
torch.cuda.synchronize()
free1 = torch.cuda.mem_get_info()[0]
ref = sim.m(3)
print(code, free0 - free1, float(np.max(np.abs(out.cpu().numpy() - ref))))
"""


def test_no_alloc_first_call_in_fresh_process():
    """In a new process that made a context on the device, the very first call
    changes the device's free memory by nothing and matches the marginal."""
    import os
    import subprocess
    import sys
    pkg = os.path.dirname(os.path.dirname(_lib.__file__))
    r = subprocess.run([sys.executable, "-c", _FIRST_CALL, pkg], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    code, dfree, err = r.stdout.split()[-3:]
    assert int(code) == 0
    assert int(dfree) == 0, f"first call took {dfree} bytes of device memory"
    assert float(err) < 1e-12


def test_no_alloc_rejects_oversized_marginal():
    sim = _state("complex128")
    bins = 1 << (QUBITS[3] + QUBITS[1])  # 16384 > 4096
    code, got = _no_alloc(sim, [3, 1], bins)
    assert code == 1
    assert "4096" in _lib.last_error()[1]
    assert np.isnan(got).all()  # output untouched
