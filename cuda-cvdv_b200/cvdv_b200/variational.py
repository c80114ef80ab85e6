"""Batched variational circuits with adjoint gradients.

A ``VariationalCircuit`` is a fixed sequence of parameterised gates on a
register layout ``[qubit registers..., mode]`` -- ``("rx", reg, qubit)`` for
Rx(theta) = exp(-i theta X / 2) and ``("cd", mode, ctrl_reg, ctrl_qubit)`` for a
conditional displacement with a real displacement beta (the reference's
``cvdvConditionalDisplacement``, src/cuda/gates.cu:163-204) -- run for many
parameter sets at once.  ``params`` is a ``(batch, n_gates)`` float64 tensor;
every instance of the batch has its own parameter for every gate.

``fidelity_loss(params, psi0, target)`` returns ``1 - |<target|psi(params)>|^2``
per instance and is differentiable in ``params``: the backward pass is the
adjoint method -- it walks the circuit backwards, applying each gate's inverse
to the final state and to the back-propagated target and reading
``g = <lambda|G|psi>`` for the gate's generator G on the way -- with the
forward states recovered by the inverse gates, not stored, and reset from a
checkpoint every ``checkpoint_every`` gates to bound the drift.  Each step is
one kernel over the whole batch (libcvdv ``cvdvBatch*``); there is no CPU
fallback.

The reference has no such form: its ``TorchCvdv`` casts gate parameters to
Python scalars, so it cannot be differentiated.
"""

from __future__ import annotations

import ctypes
from typing import List, Sequence, Tuple

import torch

from . import _lib
from .cudaCvdv import PRECISIONS, CvdvError

GateSpec = Tuple  # ("rx", reg, qubit) | ("cd", mode_reg, ctrl_reg, ctrl_qubit)


def _ptr(t: torch.Tensor) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def _check(code: int) -> None:
    if code:
        raise CvdvError(_lib.last_error(None)[1])


class VariationalCircuit:
    def __init__(self, numQubits_list: Sequence[int], gates: Sequence[GateSpec],
                 precision: str = "complex64", checkpoint_every: int = 16) -> None:
        self.qubits = list(numQubits_list)
        self.n = sum(self.qubits)
        self.mode = len(self.qubits) - 1
        self.precision = precision
        self.prec = PRECISIONS[precision]
        self.cdtype = torch.complex128 if self.prec == 0 else torch.complex64
        self.checkpoint_every = max(1, int(checkpoint_every))
        flw = [sum(self.qubits[r + 1:]) for r in range(len(self.qubits))]
        self._gates: List[Tuple[str, int]] = []
        for g in gates:
            kind = g[0]
            if kind == "rx":
                reg, k = g[1], g[2]
                self._gates.append(("rx", flw[reg] + self.qubits[reg] - 1 - k))
            elif kind == "cd":
                mode, creg, cq = g[1], g[2], g[3]
                if mode != self.mode:
                    raise ValueError("cd must act on the last register (the mode)")
                self._gates.append(("cd", flw[creg] + self.qubits[creg] - 1 - cq))
            else:
                raise ValueError(f"unsupported gate {kind!r}")
        self._L = _lib.load()

    @property
    def n_gates(self) -> int:
        return len(self._gates)

    # ---------------------------------------------------------------- kernels
    def _stream(self) -> ctypes.c_void_p:
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def _apply(self, psi: torch.Tensor, g: int, p: torch.Tensor, sign: float = 1.0) -> None:
        kind, bit = self._gates[g]
        B = psi.shape[0]
        if kind == "rx":
            _check(self._L.cvdvBatchRx(_ptr(psi), self.prec, B, self.n, bit, _ptr(p), sign, self._stream()))
        else:
            _check(self._L.cvdvBatchCondDisp(_ptr(psi), self.prec, B, self.n, self.qubits[self.mode], bit,
                                             _ptr(p), sign, self._stream()))

    def _adjoint(self, psi: torch.Tensor, lam: torch.Tensor, g: int, p: torch.Tensor) -> torch.Tensor:
        kind, bit = self._gates[g]
        B = psi.shape[0]
        out = torch.empty(2 * B, dtype=torch.float64, device=psi.device)
        if kind == "rx":
            _check(self._L.cvdvBatchRxAdjoint(_ptr(psi), _ptr(lam), self.prec, B, self.n, bit, _ptr(p),
                                              _ptr(out), self._stream()))
        else:
            _check(self._L.cvdvBatchCondDispAdjoint(_ptr(psi), _ptr(lam), self.prec, B, self.n,
                                                    self.qubits[self.mode], bit, _ptr(p), _ptr(out),
                                                    self._stream()))
        return torch.view_as_complex(out.view(B, 2))

    def _overlap(self, psi: torch.Tensor, target: torch.Tensor) -> torch.Tensor:
        B = psi.shape[0]
        out = torch.empty(2 * B, dtype=torch.float64, device=psi.device)
        per = 1 if target.dim() == 2 else 0
        _check(self._L.cvdvBatchOverlap(_ptr(psi), _ptr(target), self.prec, B, self.n, per, _ptr(out),
                                        self._stream()))
        return torch.view_as_complex(out.view(B, 2))

    # ---------------------------------------------------------------- public
    def _prepare(self, params: torch.Tensor, psi0: torch.Tensor) -> Tuple[torch.Tensor, torch.Tensor]:
        if params.dim() != 2 or params.shape[1] != self.n_gates:
            raise ValueError(f"params must be (batch, {self.n_gates})")
        B = params.shape[0]
        # gate-major copy: the parameters of one gate are contiguous for its kernel
        p = params.detach().to(device="cuda", dtype=torch.float64).t().contiguous()
        psi0 = psi0.to(device="cuda", dtype=self.cdtype)
        if psi0.shape[-1] != 1 << self.n or psi0.dim() not in (1, 2):
            raise ValueError(f"psi0 must be (2^{self.n},) or (batch, 2^{self.n})")
        psi = psi0.unsqueeze(0).expand(B, -1).contiguous() if psi0.dim() == 1 else psi0.clone()
        return p, psi

    def states(self, params: torch.Tensor, psi0: torch.Tensor) -> torch.Tensor:
        """Final states (batch, 2^n) for every parameter set; psi0 is one state or one per instance."""
        p, psi = self._prepare(params, psi0)
        for g in range(self.n_gates):
            self._apply(psi, g, p[g])
        return psi

    def fidelity_loss(self, params: torch.Tensor, psi0: torch.Tensor, target: torch.Tensor) -> torch.Tensor:
        """1 - |<target|psi_b>|^2 for every instance b (float64, differentiable in params)."""
        return _FidelityLoss.apply(params, self, psi0, target)


class _FidelityLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, params: torch.Tensor, circ: VariationalCircuit, psi0: torch.Tensor,
                target: torch.Tensor) -> torch.Tensor:
        p, psi = circ._prepare(params, psi0)
        tgt = target.to(device="cuda", dtype=circ.cdtype).contiguous()
        checkpoints = {}
        for g in range(circ.n_gates):
            if g % circ.checkpoint_every == 0 and g > 0:
                checkpoints[g] = psi.clone()  # the state before gate g
            circ._apply(psi, g, p[g])
        ov = circ._overlap(psi, tgt)
        ctx.circ = circ
        ctx.checkpoints = checkpoints
        ctx.save_for_backward(p, psi, ov, tgt)
        ctx.params_device = params.device
        return (1.0 - ov.abs() ** 2).to(params.device)

    @staticmethod
    def backward(ctx, grad_loss: torch.Tensor):
        circ: VariationalCircuit = ctx.circ
        p, psi_final, ov, tgt = ctx.saved_tensors
        B = psi_final.shape[0]
        psi = psi_final.clone()
        lam = tgt.expand(B, -1).contiguous() if tgt.dim() == 1 else tgt.clone()
        grads = torch.empty(circ.n_gates, B, dtype=torch.float64, device=psi.device)
        for g in reversed(range(circ.n_gates)):
            gval = circ._adjoint(psi, lam, g, p[g])
            # dL/dp = -2 Re(conj(ov) i <lam|G|psi>) = 2 Im(conj(ov) g)
            grads[g] = 2.0 * (ov.conj() * gval).imag
            ck = ctx.checkpoints.get(g)
            if ck is not None:
                psi.copy_(ck)
        gl = grad_loss.to(device=psi.device, dtype=torch.float64)
        return (grads.t() * gl[:, None]).to(ctx.params_device), None, None, None


def layered_gates(layers: int = 40) -> List[GateSpec]:
    """Gates of a [1, mode] circuit: `layers` x (Rx(theta_l) on the qubit, cd(beta_l) controlled by it)."""
    gates: List[GateSpec] = []
    for _ in range(layers):
        gates += [("rx", 0, 0), ("cd", 1, 0, 0)]
    return gates
