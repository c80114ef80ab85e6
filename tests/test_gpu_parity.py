"""Parity of the CUDA path (through the C ABI) with the oracle and with the
reference's own outputs (golden fixtures from TorchCvdv).

Tolerances: the plain complex128 form must match to 1e-10 relative (state L2)
and 1e-12 absolute on marginals / phase-space values; the complex64 form to
2e-5 relative.
"""

import math
import os

import numpy as np
import pytest
import torch

from oracle.cvdv_oracle import OracleSim
from tests.golden.cases import GATE_CASES

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GATES = dict(np.load(os.path.join(GOLD, "gates.npz")))
READ = dict(np.load(os.path.join(GOLD, "readouts.npz")))
C1 = dict(np.load(os.path.join(GOLD, "c1.npz")))
TORCH_DIVERGES = {"q1q2_rev"}  # see tests/test_oracle_golden.py
PLAIN_TOL = 1e-10
MIXED_TOL = 2e-5


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def make(qubits, psi, precision="complex128"):
    from cvdv_b200 import CudaCvdv
    sim = CudaCvdv(list(qubits), precision=precision, check_errors=True)
    sim.initFromArray(psi)
    return sim


def oracle(qubits, psi):
    o = OracleSim(list(qubits))
    o.set_state(psi)
    return o


def run(sim, seq):
    for meth, args in seq:
        getattr(sim, meth)(*args)


@pytest.mark.parametrize("name,qubits,seq", GATE_CASES, ids=[c[0] for c in GATE_CASES])
def test_gate_plain(name, qubits, seq):
    psi = GATES[f"{name}__in"]
    sim = make(qubits, psi)
    run(sim, seq)
    out = sim.getState()
    o = oracle(qubits, psi)
    run(o, seq)
    assert rel(out, o.get_state()) < PLAIN_TOL, name
    if name not in TORCH_DIVERGES:
        assert rel(out, GATES[f"{name}__out"]) < PLAIN_TOL, name


@pytest.mark.parametrize("name,qubits,seq", GATE_CASES, ids=[c[0] for c in GATE_CASES])
def test_gate_mixed(name, qubits, seq):
    psi = GATES[f"{name}__in"]
    sim = make(qubits, psi, "complex64")
    run(sim, seq)
    o = oracle(qubits, psi)
    run(o, seq)
    assert rel(sim.getState(), o.get_state()) < MIXED_TOL, name


def test_c1_circuit():
    from cvdv_b200 import CudaCvdv, SeparableState
    sep = SeparableState([1, 10])  # cuda tensors, as the reference
    sep.setZero(0)
    sep.setCoherent(1, 2 + 1j)
    np.testing.assert_allclose(sep.register_arrays[1].cpu().numpy(), C1["reg1"], atol=1e-15)
    sim = CudaCvdv([1, 10], check_errors=True)
    sim.initStateVector(sep)
    for meth, args in [("h", (0, 0)), ("cd", (1, 0, 0, 1.5)), ("r", (1, 0.3)), ("s", (1, 0.2)), ("h", (0, 0))]:
        getattr(sim, meth)(*args)
    assert rel(sim.getState(), C1["state"]) < PLAIN_TOL
    np.testing.assert_allclose(sim.m(0), C1["m0"], atol=1e-12)
    np.testing.assert_allclose(sim.m(1), C1["m1"], atol=1e-12)
    Wc = sim.getWigner(1, 5.0)
    assert Wc.shape == (255, 128)
    np.testing.assert_allclose(Wc, C1["wigner_b5"], atol=1e-12)
    o = OracleSim([1, 10])
    o.set_state(C1["state"])
    np.testing.assert_allclose(sim.getHusimiQ(1), o.husimi(1), atol=1e-12)
    np.testing.assert_allclose(sim.getHusimiQ(1, 5.0), C1["husimi_torch_b5"], atol=1e-6)
    np.testing.assert_allclose(sim.getHusimiQWigner(1), o.husimi_wigner(1), atol=1e-12)


def test_marginals():
    q = [2, 3, 4]
    sim = make(q, READ["m_state"])
    for key, regs in (("m_0", (0,)), ("m_1", (1,)), ("m_2", (2,)), ("m_20", (2, 0)),
                      ("m_012", (0, 1, 2)), ("m_10", (1, 0))):
        np.testing.assert_allclose(sim.m(*regs), READ[key], atol=1e-14, err_msg=key)
    assert abs(sim.m() - np.sum(np.abs(READ["m_state"]) ** 2)) < 1e-13
    each = sim.mEach([0, 2])
    np.testing.assert_allclose(each[0], READ["m_0"], atol=1e-14)
    np.testing.assert_allclose(each[1], READ["m_2"], atol=1e-14)


def test_measure_multiple_ct_alias():
    """cvdvMeasureMultipleCT (the reference's cuTENSOR variant, measure.cu:125-256)
    returns the same column-major joint marginal as cvdvMeasureMultiple."""
    import ctypes
    from cvdv_b200 import _lib
    q = [2, 3, 4]
    sim = make(q, READ["m_state"])
    L = _lib.load()
    for key, regs in (("m_20", (2, 0)), ("m_012", (0, 1, 2)), ("m_1", (1,))):
        n = int(np.prod([1 << q[r] for r in regs]))
        a, b = np.zeros(n), np.zeros(n)
        rc = (ctypes.c_int * len(regs))(*regs)
        L.cvdvMeasureMultiple(sim.ctx, rc, len(regs), a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        L.cvdvMeasureMultipleCT(sim.ctx, rc, len(regs), b.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        assert sim.last_error()[0] == 0
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-15)  # same sums, other order
        shape = tuple(1 << q[r] for r in regs)
        np.testing.assert_allclose(b.reshape(shape[::-1]).T, READ[key], atol=1e-14, err_msg=key)


def test_husimi_overlap_alias():
    """cvdvGetHusimiQOverlap (bosonic.cu:140-144) is the overlap route of
    cvdvGetHusimiQ: equal to the oracle's Husimi function."""
    import ctypes
    from cvdv_b200 import _lib
    L = _lib.load()
    for q, reg, key in (([6, 1], 0, "w_state"), ([2, 5, 2], 1, "w3_state")):
        sim = make(q, READ[key])
        o = oracle(q, READ[key])
        N = 1 << q[reg]
        out = np.zeros(N * N)
        L.cvdvGetHusimiQOverlap(sim.ctx, reg, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        assert sim.last_error()[0] == 0
        np.testing.assert_allclose(out.reshape(N, N), o.husimi(reg), atol=1e-13)
        np.testing.assert_allclose(out.reshape(N, N), sim.getHusimiQ(reg), atol=1e-14)


@pytest.mark.parametrize("qubits,reg", [([1, 12], 1), ([12, 2], 0), ([2, 9, 3], 1)])
def test_husimi_overlap_rows(qubits, reg):
    """The overlap route's fused row kernel (the circulant formed on the fly, one
    pass per output row) against the oracle's restatement of the reference's route,
    up to N = 4096 and on a strided register."""
    rng = np.random.default_rng(sum(qubits) + reg)
    n = sum(qubits)
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    psi /= np.linalg.norm(psi)
    sim = make(qubits, psi)
    o = oracle(qubits, psi)
    ref = o.husimi(reg)
    got = sim.getHusimiQ(reg)
    assert np.abs(got - ref).max() < 1e-12 * max(1.0, np.abs(ref).max())
    np.testing.assert_allclose(make(qubits, psi, "complex64").getHusimiQ(reg), ref, atol=2e-5 * np.abs(ref).max())


def test_large_marginal_global_path():
    """> 4096 bins uses the global-atomic path."""
    rng = np.random.default_rng(5)
    q = [7, 6, 2]
    psi = rng.standard_normal(1 << 15) + 1j * rng.standard_normal(1 << 15)
    psi /= np.linalg.norm(psi)
    sim = make(q, psi)
    o = oracle(q, psi)
    np.testing.assert_allclose(sim.m(0, 1), o.m(0, 1), atol=1e-14)
    np.testing.assert_allclose(sim.m(2, 0, 1), o.m(2, 0, 1), atol=1e-14)


def test_photon_number_and_state_untouched():
    sim = make([7], READ["n_state"])
    before = sim.getState()
    assert abs(sim.getPhotonNumber(0) - float(READ["n_value"])) < 1e-12
    np.testing.assert_array_equal(sim.getState(), before)


def test_wigner_husimi_readouts():
    sim = make([6, 1], READ["w_state"])
    o = oracle([6, 1], READ["w_state"])
    np.testing.assert_allclose(sim.getWigner(0), READ["w_wigner"], atol=1e-13)
    np.testing.assert_allclose(sim.getHusimiQ(0), o.husimi(0), atol=1e-13)
    sim3 = make([2, 5, 2], READ["w3_state"])
    o3 = oracle([2, 5, 2], READ["w3_state"])
    np.testing.assert_allclose(sim3.getWigner(1), READ["w3_wigner"], atol=1e-13)
    np.testing.assert_allclose(sim3.getHusimiQ(1), o3.husimi(1), atol=1e-13)
    np.testing.assert_allclose(sim3.getHusimiQWigner(1), o3.husimi_wigner(1), atol=1e-13)


def test_fidelities():
    from cvdv_b200 import SeparableState
    q = [3, 6]
    sep = SeparableState(q)
    sep.setUniform(0)
    sep.setCoherent(1, 0.7 - 0.3j)
    rng = np.random.default_rng(11)
    psi = rng.standard_normal(512) + 1j * rng.standard_normal(512)
    psi /= np.linalg.norm(psi)
    sim = make(q, psi)
    o = oracle(q, psi)
    assert abs(sim.getFidelity(sep) - o.getFidelity(sep)) < 1e-14
    phi = rng.standard_normal(512) + 1j * rng.standard_normal(512)
    phi /= np.linalg.norm(phi)
    sim2 = make(q, phi)
    o2 = oracle(q, phi)
    assert abs(sim.fidelityWith(sim2) - o.fidelity_with(o2)) < 1e-14
    # across precisions
    sim3 = make(q, phi, "complex64")
    assert abs(sim.fidelityWith(sim3) - o.fidelity_with(o2)) < 1e-6


@pytest.mark.parametrize("qubits,reg", [([13, 3], 0), ([3, 13], 1), ([12, 2], 0), ([2, 12], 1),
                                        ([14, 1], 0), ([1, 14], 1), ([5, 11, 2], 1), ([4, 4, 4, 4], 2),
                                        ([4, 4, 4, 4], 1), ([8, 6], 0), ([5, 7, 3], 0), ([6, 9, 3], 1),
                                        ([10, 4], 0), ([16, 3], 0), ([2, 13, 5], 1)])
def test_fft_layouts(qubits, reg):
    """Single- and two-pass transforms on contiguous, inner and outer registers."""
    rng = np.random.default_rng(sum(qubits) * 7 + reg)
    n = sum(qubits)
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    psi /= np.linalg.norm(psi)
    for prec, tol in (("complex128", PLAIN_TOL), ("complex64", MIXED_TOL)):
        sim = make(qubits, psi, prec)
        o = oracle(qubits, psi)
        sim.ftQ2P(reg)
        o.ft_q2p(reg)
        assert rel(sim.getState(), o.get_state()) < tol
        sim.d(reg, 0.3 - 0.2j)
        o.displacement(reg, 0.3, -0.2)
        sim.ftP2Q(reg)
        o.ft_p2q(reg)
        assert rel(sim.getState(), o.get_state()) < tol
        # two transforms of the same direction in one program, then an inverse-first one
        sim.ftQ2P(reg)
        sim.ftQ2P(reg)
        o.ft_q2p(reg)
        o.ft_q2p(reg)
        assert rel(sim.getState(), o.get_state()) < tol
        sim.sheer(reg, 0.1)
        sim.ftP2Q(reg)
        sim.sheer(reg, -0.2)
        sim.ftQ2P(reg)
        o.phase_x2(reg, 0.1)
        o.ft_p2q(reg)
        o.phase_x2(reg, -0.2)
        o.ft_q2p(reg)
        assert rel(sim.getState(), o.get_state()) < tol


@pytest.mark.parametrize("qubits,reg", [([8, 6], 0), ([10, 4], 0), ([16, 3], 0), ([2, 13, 5], 1)])
def test_column_transform_matches_tile_passes(qubits, reg):
    """The register-resident column kernel against the shared-memory tile passes
    (fusion bit 2 off) on a strided register, with diagonal runs on both sides."""
    from cvdv_b200 import _lib
    rng = np.random.default_rng(sum(qubits) * 5 + reg)
    n = sum(qubits)
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    psi /= np.linalg.norm(psi)
    o = oracle(qubits, psi)
    o.phase_x2(reg, 0.07)
    o.ft_q2p(reg)
    o.displacement(reg, 0.4, 0.1)
    ref = o.get_state()
    for prec, tol in (("complex128", PLAIN_TOL), ("complex64", MIXED_TOL)):
        outs = {}
        for flags in (15, 7, 3):
            sim = make(qubits, psi, prec)
            sim.setFusion(flags)
            _lib.load().cvdvSetTiming(sim.ctx, 1)
            sim.sheer(reg, 0.07)
            sim.ftQ2P(reg)
            sim.d(reg, 0.4 + 0.1j)
            outs[flags] = sim.getState()
            stats = _lib.kernel_stats(sim.ctx)
            assert (stats["col"][1] > 0) == (flags != 3), (prec, flags, stats)
            assert rel(outs[flags], ref) < tol, (prec, flags)
        assert rel(outs[7], outs[3]) < tol and rel(outs[15], outs[3]) < tol


COLUMN_GATES = [("d", (1, 0.3 + 0.2j)), ("r", (1, 0.7)), ("s", (2, 0.3)), ("bs", (1, 2, 0.4)),
                ("h", (0, 0)), ("cd", (1, 0, 0, 0.5 + 0.1j)), ("cr", (2, 0, 0, 0.3)),
                ("cbs", (1, 2, 0, 0, 0.25)), ("q1q2", (1, 2, 0.1)), ("cs", (1, 0, 0, 0.2)),
                ("sheer", (2, 0.05)), ("r", (2, 2.0)), ("bs", (2, 1, -0.3)), ("d", (2, -0.2 + 0.5j)),
                ("phaseCubic", (1, 0.01)), ("r", (1, -1.4)), ("cd", (2, 0, 0, -0.3 + 0.2j))]


@pytest.mark.parametrize("qubits", [[1, 9, 8, 3], [1, 13, 8, 0], [1, 8, 13, 0], [1, 10, 9, 4], [1, 14, 3, 0],
                                    [1, 12, 5, 0], [1, 11, 3, 2], [1, 11, 2, 3]])
def test_column_programs(qubits):
    """Runs of transforms and diagonal gates on strided registers (beam splitters
    between two of them, controls from a qubit register) as one on-chip pass per
    run, against the oracle and against the same circuit with column programs off."""
    from cvdv_b200 import _lib
    qubits = [q for q in qubits if q]
    rng = np.random.default_rng(sum(qubits))
    n = sum(qubits)
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    psi /= np.linalg.norm(psi)
    o = oracle(qubits, psi)
    run(o, COLUMN_GATES)
    ref = o.get_state()
    for prec, tol in (("complex128", PLAIN_TOL), ("complex64", MIXED_TOL)):
        outs = {}
        for flags in (15, 7):
            sim = make(qubits, psi, prec)
            sim.setFusion(flags)
            _lib.load().cvdvSetTiming(sim.ctx, 1)
            run(sim, COLUMN_GATES)
            outs[flags] = sim.getState()
            stats = _lib.kernel_stats(sim.ctx)
            assert stats["col"][1] > 0, (prec, flags, stats)
            assert rel(outs[flags], ref) < tol, (prec, flags, rel(outs[flags], ref))
        assert rel(outs[15], outs[7]) < tol


def _random_multimode_circuit(rng, qubits, n_gates):
    """Gates of every kind on a layout [qubit register, mode, mode, (mode)]: single-
    and two-mode gates, controlled ones from the qubits, qubit gates, quarter turns
    (transforms and parity permutations) and half-turn beam splitters (swaps)."""
    modes = list(range(1, len(qubits)))
    seq = []
    for _ in range(n_gates):
        g = int(rng.integers(14))
        m = int(modes[rng.integers(len(modes))])
        m2 = int(modes[rng.integers(len(modes))])
        k = int(rng.integers(qubits[0]))
        th = float(rng.uniform(-np.pi, np.pi))
        a = complex(rng.normal(0, 0.5), rng.normal(0, 0.5))
        if g == 0:
            seq.append(("d", (m, a)))
        elif g == 1:
            seq.append(("r", (m, th)))
        elif g == 2:
            seq.append(("s", (m, float(rng.uniform(-0.4, 0.4)))))
        elif g == 3 and m != m2:
            seq.append(("bs", (m, m2, th if qubits[m] == qubits[m2] else th / 8)))
        elif g == 4:
            seq.append(("cd", (m, 0, k, a)))
        elif g == 5:
            seq.append(("cr", (m, 0, k, th)))
        elif g == 6 and m != m2:
            seq.append(("cbs", (m, m2, 0, k, th / 4)))
        elif g == 7:
            seq.append(("h", (0, k)))
        elif g == 8:
            seq.append(("rx", (0, k, th)))
        elif g == 9:
            seq.append(("sheer", (m, float(rng.uniform(-0.2, 0.2)))))
        elif g == 10 and m != m2:
            seq.append(("q1q2", (m, m2, float(rng.uniform(-0.1, 0.1)))))
        elif g == 11:
            seq.append(("cs", (m, 0, k, float(rng.uniform(-0.3, 0.3)))))
        elif g == 12:
            seq.append((("ftQ2P", "ftP2Q")[int(rng.integers(2))], (m,)))
        else:
            seq.append(("phaseCubic", (m, float(rng.uniform(-0.02, 0.02)))))
    return seq


@pytest.mark.parametrize("qubits", [[2, 9, 9], [1, 8, 6, 5], [2, 13, 5], [1, 5, 12], [1, 6, 14], [1, 5, 13],
                                    [2, 6, 13]])
def test_random_multimode_circuits(qubits):
    """Random circuits over several modes: the planner's look-ahead (programs that
    jump over commuting stages), column chains and row programs against the oracle,
    and against the same circuit with every queue optimisation off."""
    rng = np.random.default_rng(sum(qubits) * 13 + len(qubits))
    n = sum(qubits)
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    psi /= np.linalg.norm(psi)
    seq = _random_multimode_circuit(rng, qubits, 60)
    o = oracle(qubits, psi)
    run(o, seq)
    ref = o.get_state()
    for prec, tol in (("complex128", PLAIN_TOL), ("complex64", MIXED_TOL)):
        outs = {}
        for fusion in (True, False):
            sim = make(qubits, psi, prec)
            sim.setFusion(fusion)
            run(sim, seq)
            outs[fusion] = sim.getState()
            assert rel(outs[fusion], ref) < tol, (prec, fusion, rel(outs[fusion], ref))
        assert rel(outs[True], outs[False]) < tol


@pytest.mark.parametrize("n_qubits,mode_qubits", [(3, 10), (4, 13), (2, 14)])
def test_state_transfer_scaled(n_qubits, mode_qubits):
    """The headline circuit at reduced size, plain and mixed."""
    from cvdv_b200 import CudaCvdv
    from cvdv_b200 import workloads as W
    circ = W.state_transfer(n_qubits=n_qubits, mode_qubits=mode_qubits)
    o = OracleSim(circ["qubits"])
    o.initStateVector(W.separable_arrays(circ))
    W.apply(o, circ["prep"] + circ["gates"])
    ref = o.get_state()
    for prec, tol in (("complex128", PLAIN_TOL), ("complex64", MIXED_TOL)):
        sim = CudaCvdv(circ["qubits"], precision=prec, check_errors=True)
        sim.initStateVector(W.separable_arrays(circ, device="cuda"))
        W.apply(sim, circ["prep"] + circ["gates"])
        assert rel(sim.getState(), ref) < tol, prec
        for k in range(n_qubits):
            np.testing.assert_allclose(sim.m(k), o.m(k), atol=10 * tol)


@pytest.mark.parametrize("n_qubits,mode_qubits", [(6, 12), (5, 14)])
def test_product_formed_in_first_sequence(n_qubits, mode_qubits):
    """With the product deferred and a qubit-gate sequence first in the flush, that
    sequence forms each amplitude from the register arrays' product tables (one
    outer-product launch, no product pass): equal to the oracle and to the run
    with deferral off, in both precisions (the 2^14 mode also exercises the
    blocked product)."""
    from cvdv_b200 import CudaCvdv, _lib
    from cvdv_b200 import workloads as W
    circ = W.state_transfer(n_qubits=n_qubits, mode_qubits=mode_qubits)
    o = OracleSim(circ["qubits"])
    o.initStateVector(W.separable_arrays(circ))
    W.apply(o, circ["prep"] + circ["gates"])
    ref = o.get_state()
    for prec, tol in (("complex128", PLAIN_TOL), ("complex64", MIXED_TOL)):
        outs = {}
        for flags in (31, 15):
            sim = CudaCvdv(circ["qubits"], precision=prec, check_errors=True)
            sim.setFusion(flags)
            _lib.load().cvdvSetTiming(sim.ctx, 1)
            sim.initStateVector(W.separable_arrays(circ, device="cuda"))
            W.apply(sim, circ["prep"] + circ["gates"])
            outs[flags] = sim.getState()
            st = _lib.kernel_stats(sim.ctx)
            if flags == 31:
                assert st["init"][1] == 1 and st["seq"][1] >= 1, (prec, st)
            assert rel(outs[flags], ref) < tol, (prec, flags, rel(outs[flags], ref))
        assert rel(outs[31], outs[15]) < tol


@pytest.mark.parametrize("n_qubits,mode_qubits", [(6, 14), (5, 12), (4, 9)])
def test_marginals_after_row_program(n_qubits, mode_qubits):
    """mEach of every qubit register straight after a circuit whose flush ends with
    a row program on the mode: the program writes each row's |psi|^2 and the
    marginals come from those sums (2^14 rows on the cluster kernel, 2^12 and 2^9
    on the single-CTA one), equal to the oracle; the same readout after a state
    read (no pending work) takes the marginal pass."""
    from cvdv_b200 import CudaCvdv
    from cvdv_b200 import workloads as W
    circ = W.state_transfer(n_qubits=n_qubits, mode_qubits=mode_qubits)
    o = OracleSim(circ["qubits"])
    o.initStateVector(W.separable_arrays(circ))
    W.apply(o, circ["prep"] + circ["gates"])
    ref = [o.m(k) for k in range(n_qubits)]
    for prec, tol in (("complex128", 1e-12), ("complex64", 2e-6)):
        sim = CudaCvdv(circ["qubits"], precision=prec, check_errors=True)
        sim.initStateVector(W.separable_arrays(circ, device="cuda"))
        W.apply(sim, circ["prep"] + circ["gates"])
        each = sim.mEach(list(range(n_qubits)))
        for k in range(n_qubits):
            np.testing.assert_allclose(each[k], ref[k], atol=tol, err_msg=f"{prec} {k}")
        again = sim.mEach(list(range(n_qubits)))
        for k in range(n_qubits):
            np.testing.assert_allclose(again[k], each[k], atol=tol)


def test_transform_cancellation_matches_unfused():
    """Queue cancellation of FtP2Q/FtQ2P pairs changes nothing but rounding."""
    from cvdv_b200 import CudaCvdv, _lib
    from cvdv_b200 import workloads as W
    circ = W.state_transfer(n_qubits=4, mode_qubits=12)
    out = {}
    for fusion in (True, False):
        sim = CudaCvdv(circ["qubits"], check_errors=True, fusion=fusion)
        sim.initStateVector(W.separable_arrays(circ, device="cuda"))
        W.apply(sim, circ["prep"] + circ["gates"])
        # displacements in a row on one mode, and a mode gate in between that blocks
        sim.d(4, 0.3 + 0.1j)
        sim.d(4, -0.2 + 0.4j)
        sim.cd(4, 1, 0, 0.25)
        sim.sheer(4, 0.05)
        sim.cd(4, 2, 0, -0.15)
        out[fusion] = (sim.getState(), _lib.load().cvdvCancelledTransforms(sim.ctx))
    assert out[True][1] > 0 and out[False][1] == 0
    assert rel(out[True][0], out[False][0]) < 1e-12
    o = OracleSim(circ["qubits"])
    o.initStateVector(W.separable_arrays(circ))
    W.apply(o, circ["prep"] + circ["gates"])
    o.d(4, 0.3 + 0.1j)
    o.d(4, -0.2 + 0.4j)
    o.cd(4, 1, 0, 0.25)
    o.sheer(4, 0.05)
    o.cd(4, 2, 0, -0.15)
    assert rel(out[True][0], o.get_state()) < PLAIN_TOL


def _random_qubit_circuit(rng, qubits, n_gates):
    """Qubit gates on every qubit of every register but the last (a mode), with
    conditional displacements and mode gates in between."""
    mode = len(qubits) - 1
    sites = [(r, k) for r in range(mode) for k in range(qubits[r])]
    seq = []
    for _ in range(n_gates):
        r, k = sites[rng.integers(len(sites))]
        g = rng.integers(10)
        if g == 0:
            seq.append(("h", (r, k)))
        elif g == 1:
            seq.append(("rx", (r, k, float(rng.uniform(0, 2 * np.pi)))))
        elif g == 2:
            seq.append(("ry", (r, k, float(rng.uniform(0, 2 * np.pi)))))
        elif g == 3:
            seq.append(("rz", (r, k, float(rng.uniform(0, 2 * np.pi)))))
        elif g == 4:
            seq.append((("x", "y", "z")[rng.integers(3)], (r, k)))
        elif g == 5:
            seq.append(("sheer", (mode, float(rng.uniform(-0.3, 0.3)))))
        elif g == 6:
            seq.append(("d", (mode, complex(rng.normal(0, 0.5), rng.normal(0, 0.5)))))
        else:
            seq.append(("cd", (mode, r, k, complex(rng.normal(0, 0.5), 0.0))))
    return seq


@pytest.mark.parametrize("qubits", [[1, 1, 1, 1, 1, 1, 8], [3, 2, 7], [1, 2, 1, 3, 1, 6], [2, 2, 2, 9],
                                    [1, 2, 14], [1, 1, 1, 1, 1, 1, 1, 7], [2, 1, 2, 2, 8]])
def test_qubit_gate_sequences(qubits):
    """Chains of qubit gates run as qubit-gate sequence passes: equal to the oracle
    (plain and mixed) and to the per-gate pair path."""
    from cvdv_b200 import _lib
    rng = np.random.default_rng(sum(qubits) * 7 + len(qubits))
    n = sum(qubits)
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    psi /= np.linalg.norm(psi)
    seq = _random_qubit_circuit(rng, qubits, 60)
    o = oracle(qubits, psi)
    run(o, seq)
    ref = o.get_state()
    states = {}
    for prec, tol, flags in (("complex128", PLAIN_TOL, 3), ("complex128", PLAIN_TOL, 1),
                             ("complex64", MIXED_TOL, 3)):
        sim = make(qubits, psi, prec)
        sim.setFusion(flags)
        _lib.load().cvdvSetTiming(sim.ctx, 1)
        run(sim, seq)
        out = sim.getState()
        stats = _lib.kernel_stats(sim.ctx)
        assert rel(out, ref) < tol, (prec, flags)
        assert (stats["seq"][1] > 0) == (flags == 3), (prec, flags, stats["seq"])
        states[(prec, flags)] = out
        if prec == "complex128" and flags == 3:
            # single-pass marginals of every register, and a joint one
            each = sim.mEach(list(range(len(qubits))))
            for r, pr in enumerate(each):
                np.testing.assert_allclose(pr, o.m(r), atol=1e-13, err_msg=f"mEach {r}")
            np.testing.assert_allclose(sim.m(len(qubits) - 2, 0), o.m(len(qubits) - 2, 0), atol=1e-13)
    assert rel(states[("complex128", 3)], states[("complex128", 1)]) < 1e-12


@pytest.mark.parametrize("precision,passes", [("complex128", 3), ("complex64", 3)])
def test_state_transfer_uses_sequences(precision, passes):
    """The headline chain H . CPhaseX . Rz over 14 qubits runs as a few sequence
    passes (five qubits each) between the two
    mode transforms, with the first H moved past the forward transform."""
    from cvdv_b200 import CudaCvdv, _lib
    from cvdv_b200 import workloads as W
    circ = W.state_transfer(n_qubits=14, mode_qubits=8)
    sim = CudaCvdv(circ["qubits"], precision=precision, check_errors=True)
    sim.initStateVector(W.separable_arrays(circ, device="cuda"))
    W.apply(sim, circ["prep"])
    sim.synchronize()
    _lib.load().cvdvSetTiming(sim.ctx, 1)
    _lib.kernel_stats(sim.ctx)
    W.apply(sim, circ["gates"])
    sim.synchronize()
    st = _lib.kernel_stats(sim.ctx)
    assert st["seq"][1] == passes and st["pair"][1] == 0 and st["fft_pass"][1] == 2, st
    o = OracleSim(circ["qubits"])
    o.initStateVector(W.separable_arrays(circ))
    W.apply(o, circ["prep"] + circ["gates"])
    tol = PLAIN_TOL if precision == "complex128" else MIXED_TOL
    assert rel(sim.getState(), o.get_state()) < tol


def test_gaussian_network_scaled():
    from cvdv_b200 import CudaCvdv
    from cvdv_b200 import workloads as W
    circ = W.gaussian_network(layers=6, mode_qubits=7)
    o = OracleSim(circ["qubits"])
    o.initStateVector(W.separable_arrays(circ))
    W.apply(o, circ["prep"] + circ["gates"])
    sim = CudaCvdv(circ["qubits"], check_errors=True)
    sim.initStateVector(W.separable_arrays(circ, device="cuda"))
    W.apply(sim, circ["prep"] + circ["gates"])
    assert rel(sim.getState(), o.get_state()) < PLAIN_TOL
    np.testing.assert_allclose(sim.getWigner(0), o.wigner(0), atol=1e-12)


def test_identities_reference_core():
    """Identities of the reference's tests/test_core.py at its sizes and tolerance."""
    from cvdv_b200 import CudaCvdv, SeparableState
    rng = np.random.default_rng(3)
    for _ in range(3):
        a = complex(rng.uniform(-2, 2), rng.uniform(-2, 2))
        b = complex(rng.uniform(-2, 2), rng.uniform(-2, 2))
        sim = CudaCvdv([10])
        sep = SeparableState([10])
        sep.setFock(0, 0)
        sim.initStateVector(sep)
        sim.d(0, b)
        sim.d(0, a)
        ref = SeparableState([10])
        ref.setCoherent(0, a + b)
        assert abs(sim.getFidelity(ref) - 1) < 1e-10
    # FT eigenstates
    for n in (0, 3, 11):
        sim = CudaCvdv([10])
        sep = SeparableState([10])
        sep.setFock(0, n)
        sim.initStateVector(sep)
        sim.ftQ2P(0)
        assert abs(sim.getFidelity(sep) - 1) < 1e-10
        sim.ftP2Q(0)
        assert abs(sim.getFidelity(sep) - 1) < 1e-10
    # conditional displacement commutator
    x, y = 0.41, -0.73
    sim = CudaCvdv([1, 10])
    sep = SeparableState([1, 10])
    sep.setUniform(0)
    sep.setFock(1, 0)
    sim.initStateVector(sep)
    sim.cd(1, 0, 0, x)
    sim.d(1, 1j * y)
    sim.cd(1, 0, 0, -x)
    sim.d(1, -1j * y)
    sim.rz(0, 0, 4 * x * y)
    assert abs(sim.getFidelity(sep) - 1) < 1e-10
    # beam splitter binomial populations
    nF, th = 5, 1.3
    sim = CudaCvdv([10, 10])
    sep = SeparableState([10, 10])
    sep.setFock(0, nF)
    sep.setFock(1, 0)
    sim.initStateVector(sep)
    sim.bs(0, 1, th)
    p1, p2 = math.cos(th / 2) ** 2, math.sin(th / 2) ** 2
    for j in range(nF + 1):
        s2 = SeparableState([10, 10])
        s2.setFock(0, j)
        s2.setFock(1, nF - j)
        expect = math.comb(nF, j) * p1 ** j * p2 ** (nF - j)
        assert abs(sim.getFidelity(s2) - expect) < 1e-10
    # conditional rotation phase identity
    nF, th = 7, 2.4
    sim = CudaCvdv([1, 10])
    sep = SeparableState([1, 10])
    sep.setUniform(0)
    sep.setFock(1, nF)
    sim.initStateVector(sep)
    sim.cr(1, 0, 0, th)
    sim.rz(0, 0, th * -(2 * nF + 1))
    assert abs(sim.getFidelity(sep) - 1) < 1e-10


@pytest.mark.parametrize("qubits,pairs", [([12, 11], [(0, 1)]), ([9, 4, 10], [(0, 2), (0, 1)]),
                                          ([10, 8], [(0, 1)]), ([3, 9, 9], [(1, 2)]), ([6, 8, 4], [(1, 0)]),
                                          ([6, 5, 4], [(1, 0), (2, 0)])])
def test_standalone_diagonal_runs(qubits, pairs):
    """Bilinear, shear and cubic phases with nothing to fold them into run as one
    diagonal pass.  A thread's amplitudes differ in index bits 8-9: registers that
    miss those bits (one table load, a fixed side of a bilinear term), registers
    that contain both (a side advancing by 2^(8 - shift): the bilinear term as a
    running product) and registers that hold only one of them (per amplitude),
    against the oracle in both precisions."""
    from cvdv_b200 import _lib
    L = _lib.load()
    rng = np.random.default_rng(sum(qubits) * 5 + len(pairs))
    n = sum(qubits)
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    psi /= np.linalg.norm(psi)
    seq = [("q1q2", (a, b, 0.1 + 0.05 * k)) for k, (a, b) in enumerate(pairs)]
    seq += [("sheer", (pairs[0][0], 0.05)), ("phaseCubic", (pairs[0][1], 0.01))]
    o = oracle(qubits, psi)
    run(o, seq)
    ref = o.get_state()
    for prec, tol in (("complex128", PLAIN_TOL), ("complex64", MIXED_TOL)):
        sim = make(qubits, psi, prec)
        L.cvdvSetTiming(sim.ctx, 1)
        _lib.kernel_stats(sim.ctx)
        run(sim, seq)
        L.cvdvFlush(sim.ctx)
        stats = _lib.kernel_stats(sim.ctx)
        L.cvdvSetTiming(sim.ctx, 0)
        assert stats["diag"][1] >= 1, stats
        assert rel(sim.getState(), ref) < tol, prec


def test_errors_leave_state_untouched():
    from cvdv_b200 import CudaCvdv
    from cvdv_b200 import _lib
    rng = np.random.default_rng(1)
    psi = rng.standard_normal(64) + 0j
    sim = CudaCvdv([3, 3])
    sim.initFromArray(psi)
    L = _lib.load()
    L.cvdvDisplacement(sim.ctx, 5, 1.0, 0.0)
    code, msg = sim.last_error()
    assert code == 1 and "invalid register" in msg
    L.cvdvClearError(sim.ctx)
    L.cvdvSwapRegisters(sim.ctx, 0, 1)
    L.cvdvHadamard(sim.ctx, 0, 3)  # qubit out of range
    assert sim.last_error()[0] == 1
    L.cvdvQ1Q2Gate(sim.ctx, 1, 1, 0.3)
    assert sim.last_error()[0] == 1
    np.testing.assert_allclose(sim.getState(), np.swapaxes(psi.reshape(8, 8), 0, 1).reshape(-1))
    empty = CudaCvdv([2])
    L.cvdvHadamard(empty.ctx, 0, 0)  # before init
    assert empty.last_error()[0] == 2


def test_full_size_state_transfer_properties():
    """The 2^28-amplitude circuit: norm is conserved, qubit marginals sum to it,
    and a forward/inverse transform pair of the mode returns the state."""
    from cvdv_b200 import CudaCvdv
    from cvdv_b200 import workloads as W
    circ = W.state_transfer()
    sim = CudaCvdv(circ["qubits"], check_errors=True)
    sim.initStateVector(W.separable_arrays(circ, device="cuda"))
    W.apply(sim, circ["prep"])
    n0 = sim.m()
    assert abs(n0 - 1.0) < 1e-6
    W.apply(sim, circ["gates"])
    n1 = sim.m()
    assert abs(n1 - n0) < 1e-10
    for k in range(14):
        p = sim.m(k)
        assert abs(p.sum() - n1) < 1e-10
    # with the queue optimisations off the pair is not cancelled: both 2^14-point
    # row programs run on the full state
    from cvdv_b200 import _lib
    sim.setFusion(0)
    before = sim.stateTensor().clone()
    L = _lib.load()
    L.cvdvSetTiming(sim.ctx, 1)
    _lib.kernel_stats(sim.ctx)
    sim.ftQ2P(14)
    mid = sim.stateTensor().clone()
    sim.ftP2Q(14)
    after = sim.stateTensor()
    st = _lib.kernel_stats(sim.ctx)
    assert st["fft_pass"][1] == 2, st
    moved = float(torch.linalg.vector_norm(mid - before) / torch.linalg.vector_norm(before))
    assert moved > 0.1  # the forward transform did change the state
    del mid
    err = float(torch.linalg.vector_norm(after - before) / torch.linalg.vector_norm(before))
    assert err < 1e-12


def _separable(qubits, rng):
    from cvdv_b200 import SeparableState
    sep = SeparableState(list(qubits))
    for r, q in enumerate(qubits):
        a = rng.standard_normal(1 << q) + 1j * rng.standard_normal(1 << q)
        sep.setCoeffs(r, torch.from_numpy(a / np.linalg.norm(a)))
    return sep


def _deferral_circuit(qubits, rng, couple_modes):
    """Single-mode gates of every kind on each mode, qubit gates, then gates that
    couple registers, then more single-mode gates."""
    modes = [r for r, q in enumerate(qubits) if q >= 8]
    qregs = [r for r, q in enumerate(qubits) if q < 8]
    seq = []
    for m in modes:
        seq += [("s", (m, 0.3)), ("d", (m, complex(rng.normal(0, 0.5), rng.normal(0, 0.5)))), ("r", (m, 0.7)),
                ("sheer", (m, 0.05)), ("phaseCubic", (m, 0.01)), ("h", (m, 1)), ("p", (m,)), ("ftQ2P", (m,))]
    for qr in qregs:
        seq.append(("h", (qr, 0)))
    if qregs:
        seq.append(("cd", (modes[0], qregs[0], 0, 0.4 + 0.1j)))
    if couple_modes and len(modes) > 1:
        seq.append(("bs", (modes[0], modes[1], 0.3)))
    for m in modes:
        seq += [("d", (m, 0.2 - 0.3j)), ("ftP2Q", (m,)), ("r", (m, -0.4))]
    return seq


@pytest.mark.parametrize("qubits,couple_modes", [([1, 14], True), ([2, 12], True), ([12, 2], True),
                                                 ([9, 1, 8], True), ([1, 1, 13], True), ([8, 8], True),
                                                 ([1, 12, 8], False), ([1, 10, 9, 3], False), ([3, 11], True)])
def test_product_deferral(qubits, couple_modes):
    """Gates queued after initStateVector that act on one mode alone run on that
    mode's array before the product is formed (fusion bit 4): equal to the oracle
    and to the same circuit with deferral off, in both precisions; the modes'
    transforms ahead of the coupling gates leave the state-wide passes."""
    from cvdv_b200 import CudaCvdv, _lib
    rng = np.random.default_rng(sum(qubits) * 13 + len(qubits))
    sep = _separable(qubits, rng)
    seq = _deferral_circuit(qubits, rng, couple_modes)
    o = OracleSim(list(qubits))
    o.initStateVector(sep)
    run(o, seq)
    ref = o.get_state()
    for prec, tol in (("complex128", PLAIN_TOL), ("complex64", MIXED_TOL)):
        outs, passes = {}, {}
        for flags in (31, 15):
            sim = CudaCvdv(list(qubits), precision=prec, check_errors=True)
            sim.setFusion(flags)
            _lib.load().cvdvSetTiming(sim.ctx, 1)
            sim.initStateVector(sep)
            run(sim, seq)
            outs[flags] = sim.getState()
            st = _lib.kernel_stats(sim.ctx)
            passes[flags] = st["fft_pass"][1] + st["col"][1]
            assert st["init"][1] >= 1, (prec, flags, st)
            assert rel(outs[flags], ref) < tol, (prec, flags, rel(outs[flags], ref))
        assert rel(outs[31], outs[15]) < tol
        assert passes[31] < passes[15], (prec, passes)


def test_product_deferral_edges():
    """Readout straight after initStateVector, a second initStateVector replacing
    the first with its gates, a state read in the middle, and parity of the
    deferred path with the plain one for a separable-state fidelity."""
    from cvdv_b200 import CudaCvdv
    qubits = [1, 12]
    rng = np.random.default_rng(5)
    sep1, sep2 = _separable(qubits, rng), _separable(qubits, rng)
    o = OracleSim(qubits)
    o.initStateVector(sep1)
    sim = CudaCvdv(qubits, check_errors=True)
    sim.initStateVector(sep1)
    assert rel(sim.getState(), o.get_state()) < 1e-14
    sim.d(1, 0.5 + 0.2j)
    sim.initStateVector(sep2)  # replaces the state and drops the queued gate
    sim.s(1, 0.2)
    o2 = OracleSim(qubits)
    o2.initStateVector(sep2)
    o2.s(1, 0.2)
    mid = sim.getState()
    assert rel(mid, o2.get_state()) < PLAIN_TOL
    sim.ftQ2P(1)
    sim.cd(1, 0, 0, 0.3)
    o2.ft_q2p(1)
    o2.cd(1, 0, 0, 0.3)
    assert rel(sim.getState(), o2.get_state()) < PLAIN_TOL
    sim.initStateVector(sep1)
    sim.r(1, 0.3)
    o.r(1, 0.3)
    np.testing.assert_allclose(sim.m(0), o.m(0), atol=1e-13)
    assert abs(sim.getFidelity(sep1) - o.getFidelity(sep1)) < 1e-12


def test_mode_bits_between_paired_transforms():
    """Gates between a forward and an inverse transform of a 2^14-point mode: the
    mode may stay in the blocked order only when they read it through factor
    tables (an Rz on one of its bits); a 2x2 gate on one of its bits or a control
    inside it for a gate on another register needs the natural order."""
    qubits = [9, 1, 14]
    rng = np.random.default_rng(77)
    n = sum(qubits)
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    psi /= np.linalg.norm(psi)
    seqs = [
        [("ftQ2P", (2,)), ("h", (2, 0)), ("ftP2Q", (2,))],
        [("ftQ2P", (2,)), ("h", (1, 0)), ("h", (2, 13)), ("ftP2Q", (2,))],
        [("ftQ2P", (2,)), ("cd", (0, 2, 3, 0.4j)), ("h", (1, 0)), ("ftP2Q", (2,))],
        [("ftQ2P", (2,)), ("h", (1, 0)), ("rz", (2, 5, 0.3)), ("ftP2Q", (2,))],
    ]
    for seq in seqs:
        o = oracle(qubits, psi)
        run(o, seq)
        ref = o.get_state()
        for prec, tol in (("complex128", PLAIN_TOL), ("complex64", MIXED_TOL)):
            sim = make(qubits, psi, prec)
            run(sim, seq)
            assert rel(sim.getState(), ref) < tol, (prec, seq)


def test_device_separable_setters_match_reference_fixtures():
    """SeparableState on a CUDA device writes the register arrays with the
    generator kernel (cvdvSeparableFill); they equal the reference setters'
    output (tests/golden/separable.npz, generated by src/separable.py)."""
    from cvdv_b200 import SeparableState
    SEP = dict(np.load(os.path.join(GOLD, "separable.npz")))
    for nq in (3, 6, 10):
        sep = SeparableState([nq], device="cuda")
        checks = [("zero", lambda: sep.setZero(0)), ("uniform", lambda: sep.setUniform(0))]
        checks += [(f"coherent_{a}", (lambda a=a: sep.setCoherent(0, a))) for a in (0.0, 1.0, 1.5 + 0.8j, -0.5 + 2.0j)]
        checks += [(f"fock_{n}", (lambda n=n: sep.setFock(0, n))) for n in (0, 1, 2, 5)]
        checks += [("focks", lambda: sep.setFocks(0, [0.6, 0.8j, 0.0])),
                   ("cat", lambda: sep.setCat(0, [(2.0, 1.0), (-2.0, 1.0)]))]
        for name, setter in checks:
            setter()
            a = sep.register_arrays[0]
            assert a.is_cuda and a.dtype == torch.complex128
            key = name.replace("_", f"_{nq}_", 1) if "_" in name else f"{name}_{nq}"
            np.testing.assert_allclose(a.cpu().numpy(), SEP[key], atol=1e-14, err_msg=key)


@pytest.mark.parametrize("q,rr,alpha", [(10, 0.3, 0.0), (10, 0.3, 1.2 - 0.7j), (12, -0.4, 0.5 + 0.3j),
                                        (14, 0.45, -1.1 + 0.9j)])
def test_squeezed_setter_matches_gates(q, rr, alpha):
    """setSqueezed(r, a) is the state the squeeze and displacement gates make
    from the vacuum (setFock(0), s(r), d(a)), on the device and on the host."""
    from cvdv_b200 import CudaCvdv, SeparableState
    ref = SeparableState([q], device="cuda")
    ref.setFock(0, 0)
    sim = CudaCvdv([q], check_errors=True)
    sim.initStateVector(ref)
    sim.s(0, rr)
    sim.d(0, alpha)
    want = sim.getState()
    for dev in ("cuda", "cpu"):
        sep = SeparableState([q], device=dev)
        sep.setSqueezed(0, rr, alpha)
        got = sep.register_arrays[0].cpu().numpy()
        assert rel(got, want) < 1e-10, (dev, rel(got, want))
