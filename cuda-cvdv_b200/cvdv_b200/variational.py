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
one kernel over the whole batch (libcvdv ``cvdvBatch*``; an Rx followed by a cd
controlled by the same qubit is one fused step); there is no CPU fallback.  With ``graphs=True`` both sweeps are captured in CUDA graphs once per
shape and replayed (the per-gate launch and Python overhead dominate at the
configured sizes).

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
                 precision: str = "complex64", checkpoint_every: int = 16, graphs: bool = False) -> None:
        self.qubits = list(numQubits_list)
        # graphs=True: the forward sweep and the adjoint sweep are each captured once per
        # (batch, psi0 shape, target shape) in a CUDA graph and replayed, on buffers
        # owned by the circuit (one loss/backward pair at a time per shape)
        self.graphs = bool(graphs)
        self._plans = {}
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
        # An Rx followed by a cd controlled by the same qubit runs as one fused layer
        # (cvdvBatchRxCondDisp) when no checkpoint falls between the two: the steps
        # are (first gate, number of gates) in circuit order.
        q = self.qubits[self.mode]
        self._steps: List[Tuple[int, int]] = []
        g = 0
        while g < len(self._gates):
            pair = (g + 1 < len(self._gates) and self._gates[g][0] == "rx" and self._gates[g + 1][0] == "cd"
                    and self._gates[g][1] == self._gates[g + 1][1] and 9 <= q <= 12
                    and (g + 1) % self.checkpoint_every != 0)
            self._steps.append((g, 2 if pair else 1))
            g += 2 if pair else 1

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

    def _apply_step(self, psi: torch.Tensor, g: int, n: int, p: torch.Tensor) -> None:
        """Gates g .. g + n - 1 (n = 2: the fused Rx + cd layer)."""
        if n == 1:
            self._apply(psi, g, p[g])
            return
        _check(self._L.cvdvBatchRxCondDisp(_ptr(psi), self.prec, psi.shape[0], self.n, self.qubits[self.mode],
                                           self._gates[g][1], _ptr(p[g]), _ptr(p[g + 1]), self._stream()))

    def _adjoint_step(self, psi: torch.Tensor, lam: torch.Tensor, g: int, n: int, p: torch.Tensor,
                      gvals: torch.Tensor) -> None:
        """Adjoint of gates g + n - 1 .. g, writing their g values into gvals[g ...]."""
        if n == 1:
            self._adjoint(psi, lam, g, p[g], gvals[g])
            return
        grx = torch.view_as_real(gvals[g]).view(-1)
        gcd = torch.view_as_real(gvals[g + 1]).view(-1)
        _check(self._L.cvdvBatchRxCondDispAdjoint(_ptr(psi), _ptr(lam), self.prec, psi.shape[0], self.n,
                                                  self.qubits[self.mode], self._gates[g][1], _ptr(p[g]),
                                                  _ptr(p[g + 1]), _ptr(grx), _ptr(gcd), self._stream()))

    def _adjoint(self, psi: torch.Tensor, lam: torch.Tensor, g: int, p: torch.Tensor,
                 out: torch.Tensor = None) -> torch.Tensor:
        """g_b = <lambda_b|G|psi_b> for every instance into `out` (complex128, (B,)), with
        the gate's inverse applied to both states."""
        kind, bit = self._gates[g]
        B = psi.shape[0]
        if out is None:
            out = torch.empty(B, dtype=torch.complex128, device=psi.device)
        out = torch.view_as_real(out).view(-1)
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
        for g, n in self._steps:
            self._apply_step(psi, g, n, p)
        return psi

    def fidelity_loss(self, params: torch.Tensor, psi0: torch.Tensor, target: torch.Tensor) -> torch.Tensor:
        """1 - |<target|psi_b>|^2 for every instance b (float64, differentiable in params)."""
        if self.graphs:
            return _GraphFidelityLoss.apply(params, self, psi0, target)
        return _FidelityLoss.apply(params, self, psi0, target)

    def _plan(self, B: int, psi0: torch.Tensor, target: torch.Tensor) -> "_GraphPlan":
        key = (B, tuple(psi0.shape), tuple(target.shape))
        plan = self._plans.get(key)
        if plan is None:
            plan = _GraphPlan(self, B, psi0.shape, target.shape)
            self._plans[key] = plan
        return plan


class _FidelityLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, params: torch.Tensor, circ: VariationalCircuit, psi0: torch.Tensor,
                target: torch.Tensor) -> torch.Tensor:
        p, psi = circ._prepare(params, psi0)
        tgt = target.to(device="cuda", dtype=circ.cdtype).contiguous()
        checkpoints = {}
        for g, n in circ._steps:
            if g % circ.checkpoint_every == 0 and g > 0:
                checkpoints[g] = psi.clone()  # the state before gate g
            circ._apply_step(psi, g, n, p)
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
        gvals = torch.empty(circ.n_gates, B, dtype=torch.complex128, device=psi.device)
        for g, n in reversed(circ._steps):
            circ._adjoint_step(psi, lam, g, n, p, gvals)
            ck = ctx.checkpoints.get(g)
            if ck is not None:
                psi.copy_(ck)
        # dL/dp = -2 Re(conj(ov) i <lam|G|psi>) = 2 Im(conj(ov) g), every gate at once
        grads = 2.0 * (ov.conj()[None, :] * gvals).imag
        gl = grad_loss.to(device=psi.device, dtype=torch.float64)
        return (grads.t() * gl[:, None]).to(ctx.params_device), None, None, None


class _GraphPlan:
    """Static buffers of one (batch, psi0, target) shape and the two captured
    sweeps: forward (gates, checkpoints, overlap) and adjoint (gradients)."""

    def __init__(self, circ: VariationalCircuit, B: int, psi0_shape, tgt_shape) -> None:
        dev, cd = "cuda", circ.cdtype
        self.circ = circ
        self.p = torch.zeros(circ.n_gates, B, dtype=torch.float64, device=dev)
        self.psi0 = torch.zeros(tuple(psi0_shape), dtype=cd, device=dev)
        self.tgt = torch.zeros(tuple(tgt_shape), dtype=cd, device=dev)
        self.psi = torch.empty(B, 1 << circ.n, dtype=cd, device=dev)
        self.back = torch.empty_like(self.psi)
        self.lam = torch.empty_like(self.psi)
        self.ck = {g: torch.empty_like(self.psi)
                   for g in range(circ.checkpoint_every, circ.n_gates, circ.checkpoint_every)}
        self.grads = torch.empty(circ.n_gates, B, dtype=torch.float64, device=dev)
        self.gvals = torch.empty(circ.n_gates, B, dtype=torch.complex128, device=dev)
        self.generation = 0
        # one eager run of each sweep on a side stream (first-use set-up), then capture
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            self._forward()
            self._backward()
        torch.cuda.current_stream().wait_stream(side)
        self.forward_graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.forward_graph):
            self._forward()
        self.backward_graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.backward_graph):
            self._backward()

    def _forward(self) -> None:
        c = self.circ
        self.psi.copy_(self.psi0.expand_as(self.psi))
        for g, n in c._steps:
            if g in self.ck:
                self.ck[g].copy_(self.psi)  # the state before gate g
            c._apply_step(self.psi, g, n, self.p)
        self.ov = c._overlap(self.psi, self.tgt)

    def _backward(self) -> None:
        c = self.circ
        self.back.copy_(self.psi)
        self.lam.copy_(self.tgt.expand_as(self.lam))
        for g, n in reversed(c._steps):
            c._adjoint_step(self.back, self.lam, g, n, self.p, self.gvals)
            ck = self.ck.get(g)
            if ck is not None:
                self.back.copy_(ck)
        self.grads.copy_(2.0 * (self.ov.conj()[None, :] * self.gvals).imag)


class _GraphFidelityLoss(torch.autograd.Function):
    """_FidelityLoss on captured sweeps: the same kernels in the same order."""

    @staticmethod
    def forward(ctx, params: torch.Tensor, circ: VariationalCircuit, psi0: torch.Tensor,
                target: torch.Tensor) -> torch.Tensor:
        if params.dim() != 2 or params.shape[1] != circ.n_gates:
            raise ValueError(f"params must be (batch, {circ.n_gates})")
        psi0 = psi0.to(device="cuda", dtype=circ.cdtype)
        if psi0.shape[-1] != 1 << circ.n or psi0.dim() not in (1, 2):
            raise ValueError(f"psi0 must be (2^{circ.n},) or (batch, 2^{circ.n})")
        tgt = target.to(device="cuda", dtype=circ.cdtype)
        plan = circ._plan(params.shape[0], psi0, tgt)
        plan.p.copy_(params.detach().to(device="cuda", dtype=torch.float64).t())
        plan.psi0.copy_(psi0)
        plan.tgt.copy_(tgt)
        plan.forward_graph.replay()
        plan.generation += 1
        ctx.plan, ctx.generation = plan, plan.generation
        ctx.params_device = params.device
        return (1.0 - plan.ov.abs() ** 2).to(params.device)

    @staticmethod
    def backward(ctx, grad_loss: torch.Tensor):
        plan = ctx.plan
        if plan.generation != ctx.generation:
            raise RuntimeError("VariationalCircuit(graphs=True): another fidelity_loss of the same shape "
                               "ran before this backward; run backward first or use graphs=False")
        plan.backward_graph.replay()
        gl = grad_loss.to(device="cuda", dtype=torch.float64)
        return (plan.grads.t() * gl[:, None]).to(ctx.params_device), None, None, None


def layered_gates(layers: int = 40) -> List[GateSpec]:
    """Gates of a [1, mode] circuit: `layers` x (Rx(theta_l) on the qubit, cd(beta_l) controlled by it)."""
    gates: List[GateSpec] = []
    for _ in range(layers):
        gates += [("rx", 0, 0), ("cd", 1, 0, 0)]
    return gates
