"""Transforms of strided complex64 registers of 2^12 .. 2^14 points as DFT-matrix
products on the tensor cores (cvdvSetFusion bit 5, opt-in): parity with the oracle
and with the same circuits run with the bit off (the CUDA-core column passes), and
the tensor-core passes did run.

Tolerance: 2e-5 relative state error, as for every complex64 test, for these short
sequences; split-BF16 products carry about 3e-6 relative error per 128-point DFT
(16 significant bits against FP32's 24), so long circuits drift further than with
FP32 butterflies (test_tc_random_circuit states its own bound).
"""

import numpy as np
import pytest

from oracle.cvdv_oracle import OracleSim

pytestmark = pytest.mark.gpu

MIXED_TOL = 2e-5
TC_BIT = 32


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _state(qubits, seed):
    rng = np.random.default_rng(seed)
    n = sum(qubits)
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    return psi / np.linalg.norm(psi)


def _run(qubits, psi, seq, flags):
    from cvdv_b200 import CudaCvdv, _lib
    sim = CudaCvdv(list(qubits), precision="complex64", check_errors=True)
    sim.setFusion(flags)
    sim.initFromArray(psi)
    L = _lib.load()
    L.cvdvSetTiming(sim.ctx, 1)
    _lib.kernel_stats(sim.ctx)
    for meth, args in seq:
        getattr(sim, meth)(*args)
    out = sim.getState()
    return out, _lib.kernel_stats(sim.ctx)


LAYOUTS = [([12, 6], 0), ([13, 5], 0), ([14, 5], 0), ([1, 13, 6], 1), ([12, 12], 0), ([3, 12, 7], 1)]


@pytest.mark.parametrize("qubits,reg", LAYOUTS, ids=[f"{q}-{r}" for q, r in LAYOUTS])
def test_tc_single_transforms(qubits, reg):
    psi = _state(qubits, sum(qubits) + reg)
    for seq in ([("ftQ2P", (reg,))], [("ftP2Q", (reg,))]):
        o = OracleSim(list(qubits))
        o.set_state(psi)
        for meth, args in seq:
            getattr(o, meth)(*args)
        ref = o.get_state()
        out, st = _run(qubits, psi, seq, 31 | TC_BIT)
        assert st["col_tc"][1] == 2, st  # first and last half
        assert rel(out, ref) < MIXED_TOL, (seq, rel(out, ref))


CHAINS = [
    ([13, 6], [("d", (0, 0.4 - 0.7j))]),                       # transform, phase kick, transform
    ([13, 6], [("r", (0, 0.9)), ("s", (0, 0.3))]),             # chains of four and more
    ([12, 7], [("r", (0, 2.1)), ("d", (0, -1.1 + 0.2j))]),     # a quarter turn and more
    ([13, 6], [("bs", (0, 1, 0.45))]),                         # bilinear phases on both registers
    ([1, 13, 6], [("cd", (1, 0, 0, 0.3 + 0.5j)), ("sheer", (1, 0.02))]),  # controlled, and a lone sheer
    ([14, 5], [("s", (0, -0.2)), ("phaseCubic", (0, 0.003))]),
]


@pytest.mark.parametrize("qubits,seq", CHAINS, ids=[f"{q}-{s[0][0]}" for q, s in CHAINS])
def test_tc_transform_chains(qubits, seq):
    """Runs of transforms with diagonal runs between them: the chained passes
    (middle passes with a diagonal run between two tensor-core products)."""
    psi = _state(qubits, 7 * sum(qubits))
    o = OracleSim(list(qubits))
    o.set_state(psi)
    for meth, args in seq:
        getattr(o, meth)(*args)
    ref = o.get_state()
    out, st = _run(qubits, psi, seq, 31 | TC_BIT)
    assert st["col_tc"][1] >= 2, st
    assert rel(out, ref) < MIXED_TOL, rel(out, ref)
    off, st_off = _run(qubits, psi, seq, 31)
    assert st_off["col_tc"][1] == 0
    assert rel(out, off) < MIXED_TOL


def test_tc_not_used_in_complex128_or_short_registers():
    from cvdv_b200 import CudaCvdv, _lib
    for qubits, prec in (([13, 6], "complex128"), ([11, 6], "complex64"), ([13, 4], "complex64")):
        psi = _state(qubits, 3)
        sim = CudaCvdv(qubits, precision=prec, check_errors=True)
        sim.setFusion(31 | TC_BIT)
        sim.initFromArray(psi)
        _lib.load().cvdvSetTiming(sim.ctx, 1)
        _lib.kernel_stats(sim.ctx)
        sim.ftQ2P(0)
        sim.getState()
        assert _lib.kernel_stats(sim.ctx)["col_tc"][1] == 0, (qubits, prec)


def test_tc_random_circuit():
    """A 60-gate random multi-mode circuit with the bit on: within 1e-4 relative of
    the oracle (state infidelity about 1e-8, inside the mixed form's 1e-6)."""
    from tests.test_gpu_parity import _random_multimode_circuit
    qubits = [2, 13, 5]
    rng = np.random.default_rng(sum(qubits) * 13 + len(qubits))
    psi = _state(qubits, 11)
    seq = _random_multimode_circuit(rng, qubits, 60)
    o = OracleSim(list(qubits))
    o.set_state(psi)
    for meth, args in seq:
        getattr(o, meth)(*args)
    out, st = _run(qubits, psi, seq, 31 | TC_BIT)
    assert st["col_tc"][1] > 0
    r = rel(out, o.get_state())
    assert r < 1e-4, r
    ov = abs(np.vdot(o.get_state(), out)) ** 2 / (np.vdot(out, out).real * np.vdot(o.get_state(), o.get_state()).real)
    assert 1 - ov < 1e-6
