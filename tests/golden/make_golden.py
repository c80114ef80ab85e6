"""Generate the golden fixtures under tests/golden/ from the reference itself.

Runs the reference project's own ``TorchCvdv`` + ``SeparableState``
(``src/torchCvdv.py``, ``src/separable.py``) on the CPU in complex128 and
stores their outputs as ``.npz`` fixtures.  The reference checkout is only
needed when regenerating; the committed fixtures are what the tests read.

    python tests/golden/make_golden.py /path/to/reference
    CVDV_REFERENCE=/path/to/reference python tests/golden/make_golden.py

Every input is seeded (``numpy.random.default_rng``), so re-running this
script reproduces the fixtures bit for bit on the same library versions.
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CVDV_REFERENCE")
if not REF:
    sys.exit("usage: make_golden.py /path/to/reference  (or set CVDV_REFERENCE)")
sys.path.insert(0, REF)
sys.path.insert(0, HERE)

import torch  # noqa: E402
from src.separable import SeparableState  # noqa: E402
from src.torchCvdv import TorchCvdv  # noqa: E402

torch.set_num_threads(1)
PI = np.pi


def rand_state(rng, qubits):
    n = sum(qubits)
    v = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    return (v / np.linalg.norm(v)).astype(np.complex128)


def torch_sim(qubits, psi):
    sim = TorchCvdv(list(qubits), device="cpu", dtype=torch.cdouble)
    sim.state = torch.from_numpy(psi.copy()).reshape(sim.register_dims)
    return sim


def out_state(sim):
    return sim.state.reshape(-1).numpy().copy()


from cases import GATE_CASES  # noqa: E402


def separable_fixtures():
    out = {}
    for nq in (3, 6, 10):
        sep = SeparableState([nq], device="cpu")
        sep.setZero(0)
        out[f"zero_{nq}"] = sep.register_arrays[0].numpy()
        sep.setUniform(0)
        out[f"uniform_{nq}"] = sep.register_arrays[0].numpy()
        for a in (0.0, 1.0, 1.5 + 0.8j, -0.5 + 2.0j):
            sep.setCoherent(0, a)
            out[f"coherent_{nq}_{a}"] = sep.register_arrays[0].numpy()
        for n in (0, 1, 2, 5):
            sep.setFock(0, n)
            out[f"fock_{nq}_{n}"] = sep.register_arrays[0].numpy()
        sep.setFocks(0, [0.6, 0.8j, 0.0])
        out[f"focks_{nq}"] = sep.register_arrays[0].numpy()
        sep.setCat(0, [(2.0, 1.0), (-2.0, 1.0)])
        out[f"cat_{nq}"] = sep.register_arrays[0].numpy()
        sep.setCoeffs(0, np.arange(1 << nq) / np.linalg.norm(np.arange(1 << nq)))
        out[f"coeffs_{nq}"] = sep.register_arrays[0].numpy()
    return out


def gate_fixtures():
    rng = np.random.default_rng(1234)
    out = {}
    for name, qubits, seq in GATE_CASES:
        psi = rand_state(rng, qubits)
        sim = torch_sim(qubits, psi)
        for meth, args in seq:
            getattr(sim, meth)(*args)
        out[f"{name}__in"] = psi
        out[f"{name}__out"] = out_state(sim)
        out[f"{name}__qubits"] = np.array(qubits, dtype=np.int64)
    return out


def readout_fixtures():
    rng = np.random.default_rng(99)
    out = {}
    # marginals of a random entangled state (joint orderings, duplicates excluded)
    q = [2, 3, 4]
    psi = rand_state(rng, q)
    sim = torch_sim(q, psi)
    out["m_state"] = psi
    out["m_0"] = sim.m(0)
    out["m_1"] = sim.m(1)
    out["m_2"] = sim.m(2)
    out["m_20"] = sim.m(2, 0)
    out["m_012"] = sim.m(0, 1, 2)
    out["m_10"] = sim.m(1, 0)
    # photon number of a random state of one mode, and of a mode in a product
    q1 = [7]
    psi1 = np.zeros(128, dtype=np.complex128)
    sep = SeparableState(q1, device="cpu")
    sep.setCoherent(0, 1.2 - 0.4j)
    psi1 = sep.register_arrays[0].numpy().copy()
    sim1 = torch_sim(q1, psi1)
    out["n_state"] = psi1
    out["n_value"] = np.array(sim1.getPhotonNumber(0))
    # Wigner of an entangled two-register state (register 0 is the mode)
    q2 = [6, 1]
    sa = SeparableState([6], device="cpu")
    sa.setCoherent(0, 1.0 + 0.75j)
    pa = sa.register_arrays[0].numpy()
    sa.setCoherent(0, -(1.0 + 0.75j))
    pb = sa.register_arrays[0].numpy()
    ent = (np.stack((pa, pb), axis=1) / np.sqrt(2)).reshape(-1)
    sim2 = torch_sim(q2, ent)
    out["w_state"] = ent
    out["w_wigner"] = sim2.getWigner(0)
    out["w_husimi_torch"] = sim2.getHusimiQ(0)
    # Wigner of a random state on a middle register
    q3 = [2, 5, 2]
    psi3 = rand_state(rng, q3)
    sim3 = torch_sim(q3, psi3)
    out["w3_state"] = psi3
    out["w3_wigner"] = sim3.getWigner(1)
    out["w3_husimi_torch"] = sim3.getHusimiQ(1)
    return out


def c1_fixture():
    """Config [1,10]: qubit |0>, coherent(2+1j); H, cd(1.5), r(0.3), s(0.2), H."""
    sep = SeparableState([1, 10], device="cpu")
    sep.setZero(0)
    sep.setCoherent(1, 2 + 1j)
    sim = TorchCvdv([1, 10], device="cpu", dtype=torch.cdouble)
    sim.initStateVector(sep)
    init = out_state(sim)
    sim.h(0, 0)
    sim.cd(1, 0, 0, 1.5)
    sim.r(1, 0.3)
    sim.s(1, 0.2)
    sim.h(0, 0)
    return {
        "init": init,
        "reg0": sep.register_arrays[0].numpy(),
        "reg1": sep.register_arrays[1].numpy(),
        "state": out_state(sim),
        "m0": sim.m(0),
        "m1": sim.m(1),
        "wigner_b5": sim.getWigner(1, 5.0),
        "husimi_torch_b5": sim.getHusimiQ(1, 5.0),
    }


def main():
    np.savez_compressed(os.path.join(HERE, "separable.npz"), **separable_fixtures())
    np.savez_compressed(os.path.join(HERE, "gates.npz"), **gate_fixtures())
    np.savez_compressed(os.path.join(HERE, "readouts.npz"), **readout_fixtures())
    np.savez_compressed(os.path.join(HERE, "c1.npz"), **c1_fixture())
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
