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


def test_no_alloc_rejects_oversized_marginal():
    sim = _state("complex128")
    bins = 1 << (QUBITS[3] + QUBITS[1])  # 16384 > 4096
    code, got = _no_alloc(sim, [3, 1], bins)
    assert code == 1
    assert "4096" in _lib.last_error()[1]
    assert np.isnan(got).all()  # output untouched
