"""Batched variational circuits: forward parity with the oracle, adjoint
gradients against central finite differences and against autograd through a
differentiable complex128 torch restatement of the same gates.

The reference cannot be differentiated (TorchCvdv casts gate parameters to
Python scalars), so the gradients are pinned by finite differences of the
oracle-checked forward pass."""

import math

import numpy as np
import pytest
import torch

from oracle.cvdv_oracle import OracleSim

pytestmark = pytest.mark.gpu


def _circ(precision, layers, mode_qubits, checkpoint_every=16):
    from cvdv_b200 import workloads as W
    from cvdv_b200.variational import VariationalCircuit, layered_gates
    return VariationalCircuit([1, mode_qubits], layered_gates(layers), precision=precision,
                              checkpoint_every=checkpoint_every)


def _problem(batch, layers, mode_qubits, seed=5):
    from cvdv_b200 import workloads as W
    w = W.variational(seed=seed, batch=batch, mode_qubits=mode_qubits, layers=layers)
    psi0 = W.product_state(w["qubits"], w["init"])
    tgt = W.product_state(w["qubits"], w["target"])
    return w, torch.tensor(w["params"]), psi0, tgt


def _oracle_state(qubits, params_row, psi0):
    o = OracleSim(qubits)
    o.set_state(psi0.numpy())
    for l in range(len(params_row) // 2):
        o.rx(0, 0, float(params_row[2 * l]))
        o.cd(1, 0, 0, float(params_row[2 * l + 1]))
    return o.get_state()


@pytest.mark.parametrize("precision,tol", [("complex128", 1e-10), ("complex64", 2e-5)])
def test_forward_matches_oracle(precision, tol):
    w, params, psi0, tgt = _problem(batch=6, layers=5, mode_qubits=10)
    circ = _circ(precision, 5, 10)
    out = circ.states(params, psi0).cpu().numpy()
    for b in range(params.shape[0]):
        ref = _oracle_state(w["qubits"], params[b].numpy(), psi0)
        assert np.linalg.norm(out[b] - ref) / np.linalg.norm(ref) < tol, b
    loss = circ.fidelity_loss(params, psi0, tgt).cpu().numpy()
    ref_loss = [1 - abs(np.vdot(tgt.numpy(), _oracle_state(w["qubits"], params[b].numpy(), psi0))) ** 2
                for b in range(params.shape[0])]
    np.testing.assert_allclose(loss, ref_loss, atol=10 * tol)


def test_adjoint_matches_central_differences():
    """complex128 adjoint vs central differences (h = 1e-4) of the complex128 forward."""
    layers, mq = 8, 10
    w, params, psi0, tgt = _problem(batch=2, layers=layers, mode_qubits=mq)
    circ = _circ("complex128", layers, mq, checkpoint_every=4)
    p = params.clone().requires_grad_(True)
    circ.fidelity_loss(p, psi0, tgt).sum().backward()
    grad = p.grad.numpy()
    h = 1e-4
    P = params.shape[1]
    # every perturbed parameter set is one instance of a single batched forward
    plus = params.repeat_interleave(P, dim=0)
    minus = plus.clone()
    idx = torch.arange(P).repeat(params.shape[0])
    plus[torch.arange(plus.shape[0]), idx] += h
    minus[torch.arange(minus.shape[0]), idx] -= h
    with torch.no_grad():
        lp = circ.fidelity_loss(plus, psi0, tgt).cpu().numpy()
        lm = circ.fidelity_loss(minus, psi0, tgt).cpu().numpy()
    fd = ((lp - lm) / (2 * h)).reshape(params.shape[0], P)
    scale = np.abs(fd).max()
    assert np.abs(grad - fd).max() < 1e-6 * scale + 1e-9, np.abs(grad - fd).max() / scale


def _central_differences(circ, params, psi0, tgt, h=1e-4):
    """Central differences of the loss for every parameter of every set: all
    2 x sets x params perturbed sets in one batched forward of `circ`."""
    B, P = params.shape
    plus = params.repeat_interleave(P, dim=0)
    minus = plus.clone()
    idx = torch.arange(P).repeat(B)
    plus[torch.arange(plus.shape[0]), idx] += h
    minus[torch.arange(minus.shape[0]), idx] -= h
    with torch.no_grad():
        lp = circ.fidelity_loss(plus, psi0, tgt).cpu().numpy()
        lm = circ.fidelity_loss(minus, psi0, tgt).cpu().numpy()
    return ((lp - lm) / (2 * h)).reshape(B, P)


def test_full_config_adjoint_matches_central_differences():
    """The configured problem: 64 parameter sets of [1, 12], 40 layers (80 gates),
    checkpoints every 8 layers.  The complex128 adjoint against central differences
    (h = 1e-4) of the complex128 forward: max error within 1e-6 of the largest
    gradient; the complex64 adjoint within 1e-3 of it."""
    w, params, psi0, tgt = _problem(batch=64, layers=40, mode_qubits=12)
    fd = _central_differences(_circ("complex128", 40, 12, checkpoint_every=16), params, psi0, tgt)
    scale = np.abs(fd).max()
    assert scale > 1e-3
    for precision, tol in (("complex128", 1e-6), ("complex64", 1e-3)):
        circ = _circ(precision, 40, 12, checkpoint_every=16)
        p = params.clone().requires_grad_(True)
        circ.fidelity_loss(p, psi0, tgt).sum().backward()
        err = np.abs(p.grad.numpy() - fd).max() / scale
        assert err < tol, (precision, err)


def _torch_forward(params, psi0, layers, mq):
    """Differentiable complex128 restatement: Rx on the qubit, cd = FtP2Q exp(i beta K) FtQ2P."""
    N = 1 << mq
    j = torch.arange(N, dtype=torch.float64)
    dx = math.sqrt(2 * math.pi / N)
    x = (j - (N - 1) / 2) * dx
    th = math.pi * (N - 1) * (2 * j - N + 1) / (2 * N)
    pre = torch.exp(1j * th)
    glob = complex(np.exp(1j * math.pi * (N - 1) ** 2 / (2 * N)))
    psi = psi0.reshape(2, N).to(torch.complex128)
    for l in range(layers):
        t, b = params[2 * l], params[2 * l + 1]
        c, s = torch.cos(t / 2), torch.sin(t / 2)
        psi = torch.stack([c * psi[0] - 1j * s * psi[1], -1j * s * psi[0] + c * psi[1]])
        z = torch.tensor([1.0, -1.0], dtype=torch.float64)[:, None]
        P = torch.fft.fft(psi * pre, dim=1) * pre * glob / math.sqrt(N)
        P = P * torch.exp(1j * (-math.sqrt(2) * b) * z * x)
        Q = torch.fft.ifft(P * pre.conj() * np.conj(glob), dim=1) * math.sqrt(N) * pre.conj()
        psi = Q
    return psi.reshape(-1)


def test_adjoint_matches_torch_autograd_and_mixed_precision():
    layers, mq = 6, 10
    w, params, psi0, tgt = _problem(batch=3, layers=layers, mode_qubits=mq)
    # the restatement's forward is pinned to the oracle first
    ref = _oracle_state(w["qubits"], params[0].numpy(), psi0)
    np.testing.assert_allclose(_torch_forward(params[0], psi0, layers, mq).numpy(), ref, atol=1e-12)
    auto = []
    for b in range(params.shape[0]):
        p = params[b].clone().requires_grad_(True)
        psi = _torch_forward(p, psi0, layers, mq)
        loss = 1 - torch.abs(torch.vdot(tgt.to(torch.complex128), psi)) ** 2
        loss.backward()
        auto.append(p.grad.numpy())
    auto = np.array(auto)
    for precision, tol in (("complex128", 1e-9), ("complex64", 2e-4)):
        circ = _circ(precision, layers, mq, checkpoint_every=4)
        p = params.clone().requires_grad_(True)
        circ.fidelity_loss(p, psi0, tgt).sum().backward()
        err = np.abs(p.grad.numpy() - auto).max() / np.abs(auto).max()
        assert err < tol, (precision, err)


def test_full_config_gradient_step():
    """The configured problem: 64 parameter sets, [1, 12], 40 layers, complex64,
    checkpoints every 8 layers; gradients agree with the complex128 adjoint."""
    w, params, psi0, tgt = _problem(batch=64, layers=40, mode_qubits=12)
    grads = {}
    for precision in ("complex64", "complex128"):
        circ = _circ(precision, 40, 12, checkpoint_every=16)
        p = params.clone().requires_grad_(True)
        loss = circ.fidelity_loss(p, psi0, tgt)
        loss.sum().backward()
        assert torch.isfinite(loss).all() and (loss >= -1e-6).all() and (loss <= 1 + 1e-6).all()
        grads[precision] = p.grad.numpy()
    err = np.abs(grads["complex64"] - grads["complex128"]).max() / np.abs(grads["complex128"]).max()
    assert err < 1e-3, err


@pytest.mark.parametrize("precision,qubits,tol", [("complex128", [1, 12], 1e-13), ("complex64", [1, 12], 2e-6),
                                                   ("complex128", [2, 9], 1e-13), ("complex64", [2, 10], 2e-6)])
def test_fused_layer_matches_separate_gates(precision, qubits, tol):
    """cvdvBatchRxCondDisp equals cvdvBatchRx then cvdvBatchCondDisp, and its adjoint
    equals the cd adjoint then the Rx adjoint (states and g values), on random
    states of a batch; the control is each qubit bit in turn."""
    import ctypes
    from cvdv_b200 import _lib
    L = _lib.load()
    prec = 0 if precision == "complex128" else 1
    cdt = torch.complex128 if prec == 0 else torch.complex64
    B, n, q = 5, sum(qubits), qubits[-1]
    rng = np.random.default_rng(n)
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def rnd():
        a = rng.standard_normal((B, 1 << n)) + 1j * rng.standard_normal((B, 1 << n))
        return torch.tensor(a / np.linalg.norm(a, axis=1, keepdims=True), dtype=cdt, device="cuda")

    th = torch.tensor(rng.uniform(0, 2 * np.pi, B), dtype=torch.float64, device="cuda")
    be = torch.tensor(rng.normal(0, 0.5, B), dtype=torch.float64, device="cuda")
    for bit in range(q, n):
        psi, lam = rnd(), rnd()
        a, b = psi.clone(), psi.clone()
        assert L.cvdvBatchRx(ptr(a), prec, B, n, bit, ptr(th), 1.0, stream) == 0
        assert L.cvdvBatchCondDisp(ptr(a), prec, B, n, q, bit, ptr(be), 1.0, stream) == 0
        assert L.cvdvBatchRxCondDisp(ptr(b), prec, B, n, q, bit, ptr(th), ptr(be), stream) == 0
        torch.cuda.synchronize()
        assert float((a - b).abs().max()) < tol, bit
        pa, la, pb, lb = psi.clone(), lam.clone(), psi.clone(), lam.clone()
        gcd, grx = (torch.zeros(2 * B, dtype=torch.float64, device="cuda") for _ in range(2))
        gcd2, grx2 = (torch.zeros(2 * B, dtype=torch.float64, device="cuda") for _ in range(2))
        assert L.cvdvBatchCondDispAdjoint(ptr(pa), ptr(la), prec, B, n, q, bit, ptr(be), ptr(gcd), stream) == 0
        assert L.cvdvBatchRxAdjoint(ptr(pa), ptr(la), prec, B, n, bit, ptr(th), ptr(grx), stream) == 0
        assert L.cvdvBatchRxCondDispAdjoint(ptr(pb), ptr(lb), prec, B, n, q, bit, ptr(th), ptr(be), ptr(grx2),
                                            ptr(gcd2), stream) == 0
        torch.cuda.synchronize()
        assert float((pa - pb).abs().max()) < tol and float((la - lb).abs().max()) < tol, bit
        assert float((gcd - gcd2).abs().max()) < 10 * tol * (1 + float(gcd.abs().max())), bit
        assert float((grx - grx2).abs().max()) < 10 * tol, bit


def test_graph_replay_matches_eager():
    """graphs=True (both sweeps captured once and replayed) gives the eager losses and
    gradients, on two steps in a row with different parameters."""
    from cvdv_b200.variational import VariationalCircuit, layered_gates
    w, params, psi0, tgt = _problem(batch=8, layers=6, mode_qubits=9)
    eager = VariationalCircuit([1, 9], layered_gates(6), precision="complex128", checkpoint_every=4)
    graph = VariationalCircuit([1, 9], layered_gates(6), precision="complex128", checkpoint_every=4,
                               graphs=True)
    for step in range(2):
        p = params.double() + 0.1 * step
        out = []
        for c in (eager, graph):
            q = p.clone().requires_grad_(True)
            loss = c.fidelity_loss(q, psi0, tgt)
            loss.sum().backward()
            out.append((loss.detach().cpu(), q.grad.detach().cpu()))
        assert torch.allclose(out[0][0], out[1][0], rtol=0, atol=1e-12)
        assert torch.allclose(out[0][1], out[1][1], rtol=0, atol=1e-10)

