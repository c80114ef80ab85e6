"""SeparableState: per-register wavefunctions that seed a product state.

Same interface and formulas as the reference's ``src/separable.py`` (the input
format of ``cvdvInitFromSeparable``): register arrays are complex128 torch
tensors whose ``data_ptr()`` the C ABI reads.  The default device is CUDA as in
the reference; there the setters write the arrays with the library's generator
kernel (``cvdvSeparableFill``, one launch per setter, on torch's current
stream).  ``device='cpu'`` keeps the arrays on the host, built with the same
formulas in torch, which the library also accepts (they are copied to the
device inside the call).  ``setSqueezed`` (no reference counterpart) gives the
state the squeeze and displacement gates make from the vacuum.
"""

from __future__ import annotations

import math
from typing import List, Optional, Sequence, Tuple, Union

import torch


class SeparableState:
    """Per-register state container (separable product state)."""

    def __init__(self, numQubits_list: List[int], device: str = "cuda") -> None:
        self.device = torch.device(device)
        self.num_registers = len(numQubits_list)
        self.qubit_counts = list(numQubits_list)
        self.register_dims = [1 << n for n in numQubits_list]
        self.grid_steps = [(2.0 * math.pi / d) ** 0.5 for d in self.register_dims]
        self.register_arrays: List[Optional[torch.Tensor]] = [None] * self.num_registers

    def _fill(self, r: int, kind: int, params: Sequence[float]) -> bool:
        """Generate register r on the device (False when the arrays live on the host
        or the parameters exceed the kernel's 256)."""
        if self.device.type != "cuda" or len(params) > 256:
            return False
        import ctypes
        from . import _lib
        out = torch.empty(self.register_dims[r], dtype=torch.cdouble, device=self.device)
        arr = (ctypes.c_double * max(1, len(params)))(*[float(v) for v in params])
        stream = torch.cuda.current_stream(self.device).cuda_stream
        code = _lib.load().cvdvSeparableFill(ctypes.c_void_p(out.data_ptr()), self.qubit_counts[r], kind, arr,
                                             len(params), ctypes.c_void_p(stream))
        if code:
            raise RuntimeError(_lib.last_error(None)[1])
        self.register_arrays[r] = out
        return True

    def _x(self, r: int) -> torch.Tensor:
        """Grid x_j = (j - (N-1)/2) dx (src/separable.py:34-38)."""
        N = self.register_dims[r]
        j = torch.arange(N, dtype=torch.float64, device=self.device)
        return (j - (N - 1) * 0.5) * self.grid_steps[r]

    def _gauss(self, r: int) -> torch.Tensor:
        x = self._x(r)
        return torch.exp(-0.5 * x * x) * (math.pi ** -0.25) * (self.grid_steps[r] ** 0.5)

    def setZero(self, r: int) -> None:
        """Index-0 basis state: qubit |0>; for a mode it is a position delta at
        the grid edge, not the vacuum (src/separable.py:44-48)."""
        if self._fill(r, 0, [0]):
            return
        a = torch.zeros(self.register_dims[r], dtype=torch.cdouble, device=self.device)
        a[0] = 1.0
        self.register_arrays[r] = a

    def setCoherent(self, r: int, alpha: Union[complex, float, int]) -> None:
        """|alpha> = pi^-1/4 sqrt(dx) exp(-(x-q0)^2/2) exp(i(p0 x - p0 q0/2)),
        q0 = sqrt2 Re alpha, p0 = sqrt2 Im alpha (src/separable.py:50-61)."""
        alpha = complex(alpha)
        if self._fill(r, 2, [alpha.real, alpha.imag]):
            return
        x = self._x(r)
        q0 = math.sqrt(2.0) * alpha.real
        p0 = math.sqrt(2.0) * alpha.imag
        amp = (math.pi ** -0.25) * (self.grid_steps[r] ** 0.5) * torch.exp(-0.5 * (x - q0) ** 2)
        self.register_arrays[r] = amp * torch.exp(1j * (p0 * x - p0 * q0 / 2.0)).to(torch.cdouble)

    def setFock(self, r: int, n: int) -> None:
        """Fock |n> by the Hermite-function recurrence (src/separable.py:63-73)."""
        if self._fill(r, 3, [int(n)]):
            return
        x = self._x(r)
        prev = torch.zeros_like(x)
        cur = self._gauss(r)
        for k in range(1, n + 1):
            nxt = math.sqrt(2.0 / k) * x * cur - math.sqrt((k - 1.0) / k) * prev
            prev, cur = cur, nxt
        self.register_arrays[r] = cur.to(torch.cdouble)

    def setUniform(self, r: int) -> None:
        if self._fill(r, 1, []):
            return
        N = self.register_dims[r]
        self.register_arrays[r] = torch.ones(N, dtype=torch.cdouble, device=self.device) / math.sqrt(N)

    def setFocks(self, r: int, coeffs: Union[Sequence[complex], torch.Tensor]) -> None:
        """sum_n c_n |n> with the coefficients as given (src/separable.py:81-102)."""
        c = torch.as_tensor(coeffs if isinstance(coeffs, torch.Tensor) else list(coeffs),
                            dtype=torch.cdouble).cpu()
        if not bool(torch.any(torch.abs(c) > 1e-12)):
            self.setZero(r)
            return
        if self._fill(r, 4, [v for z in c.tolist() for v in (z.real, z.imag)]):
            return
        c = c.to(self.device)
        x = self._x(r)
        fock = [self._gauss(r)]
        if len(c) > 1:
            fock.append(math.sqrt(2.0) * x * fock[0])
            for k in range(2, len(c)):
                fock.append(math.sqrt(2.0 / k) * x * fock[k - 1] - math.sqrt((k - 1.0) / k) * fock[k - 2])
        F = torch.stack(fock[: len(c)]).to(torch.cdouble)
        self.register_arrays[r] = torch.sum(c[:, None] * F, dim=0)

    def setCoeffs(self, r: int, coeffs: Union[Sequence[complex], torch.Tensor]) -> None:
        c = coeffs if isinstance(coeffs, torch.Tensor) else torch.tensor(list(coeffs))
        self.register_arrays[r] = c.to(dtype=torch.cdouble, device=self.device)

    def setCat(self, r: int, cat_states: Sequence[Tuple[Union[complex, float], Union[complex, float]]]) -> None:
        """Normalised sum_k c_k |alpha_k> (src/separable.py:113-132)."""
        pars = []
        for a, cf in cat_states:
            a, cf = complex(a), complex(cf)
            pars += [a.real, a.imag, cf.real, cf.imag]
        if self._fill(r, 5, pars):
            return
        x = self._x(r)
        psi = torch.zeros(self.register_dims[r], dtype=torch.cdouble, device=self.device)
        for a, cf in cat_states:
            a = complex(a)
            q0 = math.sqrt(2.0) * a.real
            p0 = math.sqrt(2.0) * a.imag
            coh = (math.pi ** -0.25) * (self.grid_steps[r] ** 0.5) * torch.exp(-0.5 * (x - q0) ** 2)
            psi = psi + complex(cf) * coh * torch.exp(1j * (p0 * x - p0 * q0 / 2.0)).to(torch.cdouble)
        self.register_arrays[r] = psi / torch.sqrt(torch.sum(torch.abs(psi) ** 2))

    def setSqueezed(self, r: int, rr: float, alpha: Union[complex, float, int] = 0.0) -> None:
        """(addition) D(alpha) S(rr)|0> as this library's squeeze and displacement
        gates make it from the vacuum: (e^{2 rr}/pi)^{1/4} sqrt(dx)
        exp(-e^{2 rr} (x - q0)^2 / 2) exp(i p0 (x - q0)); rr > 0 narrows |psi(x)|^2."""
        alpha = complex(alpha)
        if self._fill(r, 6, [float(rr), alpha.real, alpha.imag]):
            return
        x = self._x(r)
        q0 = math.sqrt(2.0) * alpha.real
        p0 = math.sqrt(2.0) * alpha.imag
        e2r = math.exp(2.0 * float(rr))
        amp = (e2r / math.pi) ** 0.25 * (self.grid_steps[r] ** 0.5) * torch.exp(-0.5 * e2r * (x - q0) ** 2)
        self.register_arrays[r] = amp * torch.exp(1j * (p0 * (x - q0))).to(torch.cdouble)

    def validate(self) -> None:
        for i, a in enumerate(self.register_arrays):
            if a is None:
                raise RuntimeError(f"Register {i} not initialized in SeparableState")
            if a.dtype != torch.cdouble or not a.is_contiguous() or a.numel() != self.register_dims[i]:
                raise RuntimeError(f"Register {i}: expected a contiguous complex128 array of {self.register_dims[i]}")
