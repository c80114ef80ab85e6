"""Batched independent circuits of uneven layouts: every instance of a batch run
(one persistent launch per gate stage) equals the oracle run of that instance."""

import numpy as np
import pytest
import torch

from oracle.cvdv_oracle import OracleSim

pytestmark = pytest.mark.gpu


def _oracle(inst, psi0):
    o = OracleSim(inst["qubits"])
    o.set_state(psi0.numpy())
    for name, args in inst["gates"]:
        getattr(o, name)(*args)
    return o.get_state()


def _initial(inst):
    from cvdv_b200 import workloads as W
    return W.product_state(inst["qubits"], inst["init"])


@pytest.mark.parametrize("precision,tol", [("complex64", 2e-5), ("complex128", 1e-10)])
def test_batched_instances_match_oracle(precision, tol):
    from cvdv_b200.batch import BatchedCircuits, random_instances
    insts = random_instances(seed=4, count=20, gates=14, m_range=(8, 11))
    # every mode gate kind and the quarter-turn rotations appear
    insts[0]["gates"] = [("r", (insts[0]["qubits"].__len__() - 1, a)) for a in (1.5708, 3.14159, 4.7124, 0.2)]
    insts[1]["gates"] += [("sheer", (len(insts[1]["qubits"]) - 1, 0.07)), ("ry", (0, 0, 0.4)),
                          ("ftQ2P", (len(insts[1]["qubits"]) - 1,)), ("ftP2Q", (len(insts[1]["qubits"]) - 1,))]
    B = BatchedCircuits(insts, precision=precision)
    psi0 = [_initial(i) for i in insts]
    B.set_initial(psi0)
    B.run()
    for k, inst in enumerate(insts):
        ref = _oracle(inst, psi0[k])
        got = B.state(k).cpu().numpy()
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < tol, (k, inst["qubits"])


def test_batched_graph_replay_and_large_modes():
    """Modes of 2^12..2^14 points, CUDA-graph replay equal to the direct launches, autotuned tiles."""
    from cvdv_b200.batch import BatchedCircuits, random_instances
    insts = random_instances(seed=9, count=12, gates=10, m_range=(12, 14))
    psi0 = [_initial(i) for i in insts]
    B = BatchedCircuits(insts, precision="complex64")
    B.autotune()
    B.set_initial(psi0)
    B.run()
    direct = B.states.clone()
    B.set_initial(psi0)
    B.run(graph=True)   # warm-up run + capture
    B.set_initial(psi0)
    B.run(graph=True)   # replay
    torch.cuda.synchronize()
    assert torch.allclose(B.states, direct, atol=1e-6)
    for k in (0, 5, 11):
        ref = _oracle(insts[k], psi0[k])
        got = B.state(k).cpu().numpy()
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 2e-5, k


@pytest.mark.parametrize("precision,tol", [("complex64", 2e-5), ("complex128", 1e-10)])
def test_every_row_task_shape_matches_oracle(precision, tol):
    """Each amplitudes-per-thread choice the autotuner may pick (radix-8, 16 and 32
    stage schedules, rows per CTA) gives the oracle's result, for every mode length."""
    from cvdv_b200.batch import BatchedCircuits, loge_options, random_instances
    from cvdv_b200.cudaCvdv import PRECISIONS
    prec = PRECISIONS[precision]
    top = 14 if prec == 1 else 13
    insts = random_instances(seed=21, count=top - 7, gates=8, m_range=(8, 8))
    for k, inst in enumerate(insts):  # one instance per mode length 2^8 .. 2^top (same registers)
        inst["qubits"] = inst["qubits"][:-1] + [8 + k]
    psi0 = [_initial(i) for i in insts]
    refs = [_oracle(i, p) for i, p in zip(insts, psi0)]
    for pick in range(3):
        shapes = {}
        for inst in insts:
            m = inst["qubits"][-1]
            opts = loge_options(m, prec)
            shapes[m] = opts[pick % len(opts)]
        B = BatchedCircuits(insts, precision=precision, row_loge=shapes)
        B.set_initial(psi0)
        B.run()
        for k in range(len(insts)):
            got = B.state(k).cpu().numpy()
            assert np.linalg.norm(got - refs[k]) / np.linalg.norm(refs[k]) < tol, (shapes, k)
