"""CPU checks that the seeded benchmark circuits have the configured shapes.

The state transfer (14 qubit registers + a 2^14-point mode, 14 rounds of H, cd
with beta_k = sqrt(pi/2) 2^-k and Rz), the two-mode [13, 13] network (200 layers
of beam splitter, rotations and displacements), the [1, 10] qubit-mode circuit
and the [1, 12] variational batch (64 sets, 40 layers of Rx + cd).
"""

import math

import numpy as np

from cvdv_b200 import workloads as W


def test_state_transfer_configuration():
    c = W.state_transfer()
    assert c["qubits"] == [1] * 14 + [14] and sum(c["qubits"]) == 28
    g = c["gates"]
    assert len(g) == 42
    for k in range(1, 15):
        h, cd, rz = g[3 * (k - 1): 3 * k]
        assert h == ("h", (k - 1, 0))
        assert cd[0] == "cd" and cd[1][:3] == (14, k - 1, 0)
        assert math.isclose(cd[1][3], math.sqrt(math.pi / 2) * 2.0 ** (-k), rel_tol=0, abs_tol=1e-15)
        assert rz[0] == "rz" and rz[1][:2] == (k - 1, 0) and 0.0 <= rz[1][2] < 2 * math.pi
    (s_name, (s_reg, r)), (d_name, (d_reg, alpha)) = c["prep"]
    assert (s_name, d_name, s_reg, d_reg) == ("s", "d", 14, 14) and 0.0 <= r <= 0.5
    assert c["init"] == [("setZero", ())] * 14 + [("setFock", (0,))]
    assert c["readout"] == [("m", (k,)) for k in range(14)]
    # seeded: the same circuit every time, another seed another one
    assert W.state_transfer() == c and W.state_transfer(seed=3)["gates"] != g
    small = W.state_transfer(n_qubits=3, mode_qubits=9)
    assert small["qubits"] == [1, 1, 1, 9] and len(small["gates"]) == 9


def test_gaussian_network_configuration():
    c = W.gaussian_network()
    assert c["qubits"] == [13, 13]
    (s0, (r0a, r0)), (s1, (r1a, r1)) = c["prep"]
    assert (s0, s1, r0a, r1a) == ("s", "s", 0, 1) and 0.2 <= r0 <= 0.8 and 0.2 <= r1 <= 0.8
    g = c["gates"]
    assert len(g) == 200 * 5
    for layer in range(200):
        bs, ra, rb, da, db = g[5 * layer: 5 * layer + 5]
        assert bs[0] == "bs" and bs[1][:2] == (0, 1) and 0.0 <= bs[1][2] <= math.pi / 2
        assert (ra[0], ra[1][0], rb[0], rb[1][0]) == ("r", 0, "r", 1)
        assert 0.0 <= ra[1][1] < 2 * math.pi and 0.0 <= rb[1][1] < 2 * math.pi
        assert (da[0], da[1][0], db[0], db[1][0]) == ("d", 0, "d", 1)
    assert c["readout"] == [("m", (0,)), ("m", (1,)), ("getWigner", (0,))]


def test_qubit_mode_configuration():
    c = W.qubit_mode()
    assert c["qubits"] == [1, 10]
    assert c["init"] == [("setZero", ()), ("setCoherent", (2 + 1j,))]
    assert c["gates"] == [("h", (0, 0)), ("cd", (1, 0, 0, 1.5)), ("r", (1, 0.3)), ("s", (1, 0.2)),
                          ("h", (0, 0))]


def test_variational_configuration():
    c = W.variational()
    assert c["qubits"] == [1, 12]
    p = c["params"]
    assert p.shape == (64, 80)
    theta, beta = p[:, 0::2], p[:, 1::2]
    assert theta.min() >= 0.0 and theta.max() < 2 * math.pi
    assert abs(beta.mean()) < 0.1 and 0.4 < beta.std() < 0.6
    assert c["gates"] == [("rx", (0, 0)), ("cd", (1, 0, 0))] * 40


def test_product_state_is_the_register_outer_product():
    psi = W.product_state([1, 3], [("setZero", ()), ("setCoherent", (0.5 + 0.2j,))]).numpy()
    from cvdv_b200.separable import SeparableState
    sep = SeparableState([1, 3], device="cpu")
    sep.setZero(0)
    sep.setCoherent(1, 0.5 + 0.2j)
    ref = np.kron(sep.register_arrays[0].numpy(), sep.register_arrays[1].numpy())
    np.testing.assert_allclose(psi, ref, atol=1e-15)
    assert psi.shape == (16,) and abs(psi[8:]).max() == 0.0  # qubit |0>: the upper half is empty
