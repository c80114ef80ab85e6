"""CPU checks of the batched-circuit compiler (``cvdv_b200.batch``).

``BatchedCircuits`` compiles each gate, on the host, into a row-program record
(diagonal phase runs, unnormalised transforms, parity) or a 2x2 matrix, which the
stage kernel then runs.  These tests run the compiled records through a numpy
interpreter with the stage kernel's semantics (``csrc/kernels_stage.cu``:
``phase_factor`` and ``stage_row_task``) and compare each gate with the oracle,
so the host-side decompositions are checked without a GPU.
"""

import math

import numpy as np
import pytest

from cvdv_b200.batch import (OP_DIAG, OP_FWD, OP_INV, OP_PARITY, PROGRAM_DTYPE, _mode_program,
                             _qubit_matrix, _RowProgram, loge_options)
from oracle.cvdv_oracle import OracleSim

Q = 8
N = 1 << Q


def phase_factor(P, N, zs):
    """The stage kernel's diagonal factor of one run, on every point of a row."""
    j = np.arange(N, dtype=np.int64)
    m = ((N - 1) * (2 * j - N + 1)) % (4 * N)
    m = (m * int(P["tw"])) % (4 * N)
    dx = math.sqrt(2.0 * math.pi / N)
    x = (j - 0.5 * (N - 1)) * dx
    ph = (math.pi * m / (2 * N) + P["g0"] + zs * P["h0"]
          + x * ((P["a1"] + zs * P["b1"]) + x * ((P["a2"] + zs * P["b2"]) + x * P["a3"])))
    return P["scale"] * np.exp(1j * ph)


def run_record(rec, v, zs):
    """Apply a compiled program record to one row (zs = -1 where its control bit is set)."""
    v = v.astype(np.complex128).copy()
    d = 0
    for op in rec["op"][: int(rec["nOps"])]:
        if op == OP_DIAG:
            P = rec["phase"][d]
            d += 1
            v = v * phase_factor(P, len(v), zs if int(P["ctrlBit"]) >= 0 else 1.0)
        elif op == OP_FWD:
            v = np.fft.fft(v)
        elif op == OP_INV:
            v = np.fft.ifft(v) * len(v)
        elif op == OP_PARITY:
            v = v[::-1].copy()
        else:
            raise AssertionError(f"unknown op {op}")
    return v


def random_state(rng, n):
    psi = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    return psi / np.linalg.norm(psi)


MODE_GATES = [("d", (0.7 - 0.4j,)), ("d", (1e-13 + 0.3j,)), ("d", (-1.1 + 0j,)), ("s", (0.35,)), ("s", (-0.2,)),
              ("sheer", (0.04,)), ("ftQ2P", ()), ("ftP2Q", ()), ("r", (0.3,)), ("r", (1.9,)), ("r", (3.3,)),
              ("r", (-1.4,)), ("r", (math.pi / 2,)), ("r", (0.0,))]


@pytest.mark.parametrize("name,args", MODE_GATES, ids=[f"{g}{a}" for g, a in MODE_GATES])
def test_mode_gate_programs_match_oracle(name, args):
    rng = np.random.default_rng(abs(hash((name, args))) % (2 ** 32))
    psi = random_state(rng, N)
    o = OracleSim([Q])
    o.set_state(psi)
    getattr(o, name)(0, *args)
    rec = _mode_program(name, args, N, -1).record()
    out = run_record(rec, psi, 1.0)
    np.testing.assert_allclose(out, o.get_state(), atol=1e-12)


@pytest.mark.parametrize("alpha", [0.8 + 0.0j, 0.5 - 0.6j, 0.0 + 0.9j])
def test_conditional_displacement_program_matches_oracle(alpha):
    """cd on a [1, Q] layout: the qubit (flat bit Q) selects zs = +1 / -1 per row."""
    rng = np.random.default_rng(7)
    psi = random_state(rng, 2 * N)
    o = OracleSim([1, Q])
    o.set_state(psi)
    o.cd(1, 0, 0, alpha)
    rec = _mode_program("cd", (alpha,), N, Q).record()
    out = np.concatenate([run_record(rec, psi[:N], 1.0), run_record(rec, psi[N:], -1.0)])
    np.testing.assert_allclose(out, o.get_state(), atol=1e-12)


def test_rz_row_phase_and_qubit_matrices_match_oracle():
    """Rz as a row phase on the qubit's bit (h0 = -theta / 2), H / Rx / Ry as 2x2 matrices."""
    rng = np.random.default_rng(3)
    psi = random_state(rng, 2 * N)
    th = 0.83
    o = OracleSim([1, Q])
    o.set_state(psi)
    o.rz(0, 0, th)
    P = _RowProgram(N)
    ph = P._diag()
    ph.ctrl = Q
    ph.c["h0"] = -0.5 * th
    rec = P.record()
    out = np.concatenate([run_record(rec, psi[:N], 1.0), run_record(rec, psi[N:], -1.0)])
    np.testing.assert_allclose(out, o.get_state(), atol=1e-12)
    for name, args in (("h", (0, 0)), ("rx", (0, 0, 0.61)), ("ry", (0, 0, -1.2))):
        o = OracleSim([1, Q])
        o.set_state(psi)
        getattr(o, name)(*args)
        M = _qubit_matrix(name, args).reshape(2, 2)
        out = np.tensordot(M, psi.reshape(2, N), axes=(1, 0)).reshape(-1)
        np.testing.assert_allclose(out, o.get_state(), atol=1e-12)
    assert _qubit_matrix("rz", (0, 0, th)) is None


def test_program_record_limits_and_row_shapes():
    P = _RowProgram(N)
    for _ in range(8):
        P.ft(1)
        P.ft(-1)
    with pytest.raises(ValueError):
        P.record()
    rec = _mode_program("s", (0.3,), N, -1).record()
    assert int(rec["nOps"]) == 9 and rec.dtype == PROGRAM_DTYPE
    # a row task's amplitudes per thread: the row fits 512 threads; complex128 at most 16
    assert loge_options(8, 0) == [3, 4] and loge_options(14, 1) == [5]
    assert loge_options(13, 0) == [4] and loge_options(12, 1) == [3, 4, 5]
