"""CPU checks of VariationalCircuit's step plan: which Rx + cd pairs run as one
fused layer (no GPU call is made)."""

import pytest

from cvdv_b200.variational import VariationalCircuit, layered_gates


def _steps(qubits, gates, ce):
    return VariationalCircuit(qubits, gates, checkpoint_every=ce)._steps


def test_layers_fuse_into_pairs():
    steps = _steps([1, 12], layered_gates(40), 16)
    assert steps == [(2 * l, 2) for l in range(40)]


def test_no_pair_across_a_checkpoint():
    # checkpoints every 3 gates: the pair starting at gate 2 would end on gate 3
    steps = _steps([1, 10], layered_gates(4), 3)
    covered = [g for g, n in steps for g in range(g, g + n)]
    assert covered == list(range(8))
    for g, n in steps:
        if n == 2:
            assert (g + 1) % 3 != 0
    assert (2, 1) in steps and (3, 1) in steps


@pytest.mark.parametrize("mode_qubits,fused", [(8, False), (9, True), (12, True)])
def test_fusion_needs_rows_of_at_least_512_points(mode_qubits, fused):
    steps = _steps([1, mode_qubits], layered_gates(2), 16)
    assert all(n == (2 if fused else 1) for _, n in steps)


def test_control_must_be_the_rotated_qubit():
    gates = [("rx", 0, 0), ("cd", 2, 1, 0), ("rx", 1, 0), ("cd", 2, 1, 0)]
    steps = _steps([1, 1, 10], gates, 16)
    assert steps == [(0, 1), (1, 1), (2, 2)]
