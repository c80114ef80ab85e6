"""Seeded synthetic circuits for the benchmark configurations.

A circuit is ``(qubits, init, prep, gates, readout)``: ``init`` lists one
separable-state setter per register, ``prep`` and ``gates`` are lists of
``(method, args)`` in the ``CudaCvdv`` API, ``readout`` lists the readouts.
Only ``gates`` is timed as "the circuit"; ``prep`` builds the input state.
All random draws come from ``numpy.random.default_rng(seed)`` in gate order.

* ``state_transfer`` -- CV-to-DV state transfer, 14 qubit registers + one mode
  of 2^14 points (2^28 amplitudes): per round k = 1..14, H on qubit k-1,
  cd(beta_k = sqrt(pi/2) 2^-k) controlled by it, Rz(phi_k), phi_k ~ U[0, 2pi).
  The mode starts in D(alpha) S(r) |0>, r ~ U[0, 0.5], alpha = 1.5 (X + iY)/sqrt2
  with X, Y ~ N(0,1) (sigma 1.5 per complex amplitude); the qubits in |0>.
  Readout: the marginal of every qubit register.  ``n_qubits`` / ``mode_qubits``
  scale it down for tests.
* ``gaussian_network`` -- two modes [13, 13] (2^26): squeezed vacua r ~ U[0.2, 0.8];
  layers of bs(theta ~ U[0, pi/2]), r(phi ~ U[0, 2pi)) on each mode, d(alpha) on
  each mode with alpha = (X + iY)/sqrt2, X, Y ~ N(0,1).  Readout: both position
  marginals and the Wigner function of mode 0.
* ``qubit_mode`` -- [1, 10]: qubit |0>, coherent(2+1j); H, cd(1.5), r(0.3),
  s(0.2), H.  Readout: state, both marginals, Wigner of the mode.
* ``variational`` -- [1, 12], a batch of 64 parameter sets: 40 layers of
  (Rx(theta_l) on the qubit, cd(beta_l) controlled by it), theta ~ U[0, 2pi),
  beta ~ N(0, 0.5) real.  Start: qubit |0> x mode vacuum (the configuration names
  no start state; the vacuum is the choice here).  Target: qubit |0> x the
  normalised even cat |2> + |-2>.  Loss 1 - |<target|psi>|^2.
"""

from __future__ import annotations

import math
from typing import Any, Dict, List, Tuple

import numpy as np

Gate = Tuple[str, tuple]


def state_transfer(seed: int = 2, n_qubits: int = 14, mode_qubits: int = 14) -> Dict[str, Any]:
    rng = np.random.default_rng(seed)
    r_sq = float(rng.uniform(0.0, 0.5))
    alpha = complex(1.5 * (rng.standard_normal() + 1j * rng.standard_normal()) / math.sqrt(2.0))
    mode = n_qubits
    qubits = [1] * n_qubits + [mode_qubits]
    init = [("setZero", ())] * n_qubits + [("setFock", (0,))]
    prep: List[Gate] = [("s", (mode, r_sq)), ("d", (mode, alpha))]
    gates: List[Gate] = []
    for k in range(1, n_qubits + 1):
        phi = float(rng.uniform(0.0, 2.0 * math.pi))
        beta = math.sqrt(math.pi / 2.0) * 2.0 ** (-k)
        gates += [("h", (k - 1, 0)), ("cd", (mode, k - 1, 0, beta)), ("rz", (k - 1, 0, phi))]
    readout = [("m", (k,)) for k in range(n_qubits)]
    return dict(name="state_transfer", qubits=qubits, init=init, prep=prep, gates=gates,
                readout=readout, seed=seed)


def gaussian_network(seed: int = 3, layers: int = 200, mode_qubits: int = 13) -> Dict[str, Any]:
    rng = np.random.default_rng(seed)
    qubits = [mode_qubits, mode_qubits]
    r0 = float(rng.uniform(0.2, 0.8))
    r1 = float(rng.uniform(0.2, 0.8))
    init = [("setFock", (0,)), ("setFock", (0,))]
    prep: List[Gate] = [("s", (0, r0)), ("s", (1, r1))]
    gates: List[Gate] = []
    for _ in range(layers):
        th = float(rng.uniform(0.0, math.pi / 2))
        p0 = float(rng.uniform(0.0, 2 * math.pi))
        p1 = float(rng.uniform(0.0, 2 * math.pi))
        a0 = complex((rng.standard_normal() + 1j * rng.standard_normal()) / math.sqrt(2.0))
        a1 = complex((rng.standard_normal() + 1j * rng.standard_normal()) / math.sqrt(2.0))
        gates += [("bs", (0, 1, th)), ("r", (0, p0)), ("r", (1, p1)), ("d", (0, a0)), ("d", (1, a1))]
    readout = [("m", (0,)), ("m", (1,)), ("getWigner", (0,))]
    return dict(name="gaussian_network", qubits=qubits, init=init, prep=prep, gates=gates,
                readout=readout, seed=seed)


def qubit_mode() -> Dict[str, Any]:
    return dict(name="qubit_mode", qubits=[1, 10], init=[("setZero", ()), ("setCoherent", (2 + 1j,))],
                prep=[], gates=[("h", (0, 0)), ("cd", (1, 0, 0, 1.5)), ("r", (1, 0.3)), ("s", (1, 0.2)),
                                ("h", (0, 0))],
                readout=[("m", (0,)), ("m", (1,)), ("getWigner", (1,))], seed=None)


def separable_arrays(circ: Dict[str, Any], device: str = "cpu"):
    """The circuit's initial register arrays as a SeparableState."""
    from .separable import SeparableState
    sep = SeparableState(circ["qubits"], device=device)
    for r, (meth, args) in enumerate(circ["init"]):
        getattr(sep, meth)(r, *args)
    return sep


def apply(sim, gates: List[Gate]) -> None:
    """Run (method, args) pairs on any object with the CudaCvdv gate API."""
    for meth, args in gates:
        getattr(sim, meth)(*args)


def variational(seed: int = 5, batch: int = 64, mode_qubits: int = 12, layers: int = 40) -> Dict[str, Any]:
    rng = np.random.default_rng(seed)
    theta = rng.uniform(0.0, 2.0 * math.pi, size=(batch, layers))
    beta = rng.normal(0.0, 0.5, size=(batch, layers))
    params = np.empty((batch, 2 * layers))
    params[:, 0::2] = theta
    params[:, 1::2] = beta
    qubits = [1, mode_qubits]
    init = [("setZero", ()), ("setFock", (0,))]
    target = [("setZero", ()), ("setCat", ([(2.0, 1.0), (-2.0, 1.0)],))]
    gates: List[Gate] = []
    for _ in range(layers):
        gates += [("rx", (0, 0)), ("cd", (1, 0, 0))]
    return dict(name="variational", qubits=qubits, init=init, target=target, gates=gates, params=params,
                seed=seed)


def product_state(qubits, setters, device: str = "cpu"):
    """Flat state vector (complex128 torch tensor) of a separable state."""
    import torch
    from .separable import SeparableState
    sep = SeparableState(qubits, device=device)
    for r, (meth, args) in enumerate(setters):
        getattr(sep, meth)(r, *args)
    psi = sep.register_arrays[0]
    for a in sep.register_arrays[1:]:
        psi = torch.outer(psi, a).reshape(-1)
    return psi
