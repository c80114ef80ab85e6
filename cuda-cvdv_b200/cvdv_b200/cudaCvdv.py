"""CudaCvdv: the reference's Python API over the B200 libcvdv.so.

Method names, argument meaning, return shapes and the C calls behind them follow
the reference's ``src/cudaCvdv.py:77-252`` so that code written against the
reference runs unchanged.  Additions (keyword-only or new methods) are marked.
"""

from __future__ import annotations

import ctypes
from ctypes import POINTER, c_double, c_int
from typing import Any, List, Optional, Tuple

import numpy as np
import numpy.typing as npt
import torch

from . import _lib
from .separable import SeparableState

PRECISIONS = {"complex128": 0, "c128": 0, "plain": 0, "complex64": 1, "c64": 1, "mixed": 1}


class CvdvError(RuntimeError):
    pass


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(POINTER(c_double))


class CudaCvdv:
    """Dense CV-DV simulator on one GPU.  ``precision`` (addition): "complex128"
    (default, the reference's arithmetic) or "complex64" (mixed precision)."""

    def __init__(self, numQubits_list: List[int], precision: str = "complex128",
                 check_errors: bool = False, fusion: bool = True) -> None:
        self._L = _lib.load()
        self.num_registers = len(numQubits_list)
        self.register_dims = [1 << q for q in numQubits_list]
        self.total_size = int(np.prod(self.register_dims, dtype=np.int64))
        self.qubit_counts = np.array(numQubits_list, dtype=np.int32)
        self.grid_steps = np.array([np.sqrt(2 * np.pi / d) for d in self.register_dims], dtype=np.float64)
        self.precision = precision
        self.check_errors = check_errors
        q = (c_int * len(numQubits_list))(*numQubits_list)
        self.ctx = self._L.cvdvCreateEx(len(numQubits_list), q, PRECISIONS[precision])
        if not self.ctx:
            raise CvdvError("cvdvCreate failed")
        code, msg = _lib.last_error(self.ctx)
        if code:
            raise CvdvError(msg)
        self.setFusion(fusion)

    def setFusion(self, on) -> None:
        """(addition) queue optimisations, all on by default: bit 0 cancels
        FtP2Q/FtQ2P pairs separated only by gates on other registers (exact
        identity); bit 1 runs chains of qubit gates on up to five qubits as one
        pass; bit 2 transforms non-last registers with the register-resident
        column kernel; bit 3 runs transform/diagonal runs on a non-last register
        as one pass with each column on chip; bit 4 applies the gates queued
        after initStateVector that act on one mode alone (before it is coupled
        to another register) to that mode's array before the product state is
        formed; bit 5 (not in True; opt-in) runs complex64 transforms of non-last
        registers of 2^12 .. 2^14 points as DFT-matrix products on the tensor
        cores.  True = bits 0-4, False = none, an int = those bits."""
        flags = (31 if on else 0) if isinstance(on, bool) else int(on)
        self._L.cvdvSetFusion(self.ctx, flags)

    def __del__(self):
        try:
            if getattr(self, "ctx", None):
                self._L.cvdvDestroy(self.ctx)
                self.ctx = None
        except Exception:
            pass

    # -------------------------------------------------------------- errors (addition)
    def last_error(self) -> Tuple[int, str]:
        return _lib.last_error(self.ctx)

    def _check(self):
        if self.check_errors:
            code, msg = _lib.last_error(self.ctx)
            if code:
                self._L.cvdvClearError(self.ctx)
                raise CvdvError(msg)

    # -------------------------------------------------------------- init
    def initStateVector(self, sep: SeparableState) -> None:
        sep.validate()
        ptrs = (ctypes.c_void_p * self.num_registers)(
            *[ctypes.c_void_p(a.data_ptr()) for a in sep.register_arrays])
        self._L.cvdvInitFromSeparable(self.ctx, ptrs, self.num_registers)
        self._check()

    def initFromArray(self, arr) -> None:
        if isinstance(arr, torch.Tensor):
            t = arr.reshape(-1).to(dtype=torch.cdouble).contiguous()
        else:
            t = torch.from_numpy(np.ascontiguousarray(np.asarray(arr, dtype=np.complex128).reshape(-1)))
        if t.numel() != self.total_size:
            raise ValueError(f"expected {self.total_size} amplitudes, got {t.numel()}")
        self._L.cvdvSetStateFromDevicePtr(self.ctx, ctypes.c_void_p(t.data_ptr()))
        self._check()

    # -------------------------------------------------------------- gates
    def d(self, regIdx: int, beta) -> None:
        beta = complex(beta)
        self._L.cvdvDisplacement(self.ctx, regIdx, beta.real, beta.imag)
        self._check()

    def cd(self, targetReg: int, ctrlReg: int, ctrlQubit: int, alpha) -> None:
        alpha = complex(alpha)
        self._L.cvdvConditionalDisplacement(self.ctx, targetReg, ctrlReg, ctrlQubit, alpha.real, alpha.imag)
        self._check()

    def cr(self, targetReg: int, ctrlReg: int, ctrlQubit: int, theta) -> None:
        self._L.cvdvConditionalRotation(self.ctx, targetReg, ctrlReg, ctrlQubit, float(theta))
        self._check()

    def x(self, r: int, k: int) -> None: self.rx(r, k, np.pi)
    def y(self, r: int, k: int) -> None: self.ry(r, k, np.pi)
    def z(self, r: int, k: int) -> None: self.rz(r, k, np.pi)

    def rx(self, r: int, k: int, theta) -> None:
        self._L.cvdvPauliRotation(self.ctx, r, k, 0, float(theta))
        self._check()

    def ry(self, r: int, k: int, theta) -> None:
        self._L.cvdvPauliRotation(self.ctx, r, k, 1, float(theta))
        self._check()

    def rz(self, r: int, k: int, theta) -> None:
        self._L.cvdvPauliRotation(self.ctx, r, k, 2, float(theta))
        self._check()

    def h(self, r: int, k: int) -> None:
        self._L.cvdvHadamard(self.ctx, r, k)
        self._check()

    def p(self, r: int) -> None:
        self._L.cvdvParity(self.ctx, r)
        self._check()

    def cp(self, targetReg: int, ctrlReg: int, ctrlQubit: int) -> None:
        self._L.cvdvConditionalParity(self.ctx, targetReg, ctrlReg, ctrlQubit)
        self._check()

    def swap(self, r1: int, r2: int) -> None:
        self._L.cvdvSwapRegisters(self.ctx, r1, r2)
        self._check()

    def sheer(self, r: int, t) -> None:
        self._L.cvdvPhaseSquare(self.ctx, r, float(t))
        self._check()

    def phaseCubic(self, r: int, t) -> None:
        self._L.cvdvPhaseCubic(self.ctx, r, float(t))
        self._check()

    def r(self, r: int, theta) -> None:
        self._L.cvdvRotation(self.ctx, r, float(theta))
        self._check()

    def s(self, r: int, rr) -> None:
        self._L.cvdvSqueeze(self.ctx, r, float(rr))
        self._check()

    def cs(self, targetReg: int, ctrlReg: int, ctrlQubit: int, rr) -> None:
        self._L.cvdvConditionalSqueeze(self.ctx, targetReg, ctrlReg, ctrlQubit, float(rr))
        self._check()

    def bs(self, r1: int, r2: int, theta) -> None:
        self._L.cvdvBeamSplitter(self.ctx, r1, r2, float(theta))
        self._check()

    def cbs(self, r1: int, r2: int, ctrlReg: int, ctrlQubit: int, theta) -> None:
        self._L.cvdvConditionalBeamSplitter(self.ctx, r1, r2, ctrlReg, ctrlQubit, float(theta))
        self._check()

    def q1q2(self, r1: int, r2: int, coeff) -> None:
        self._L.cvdvQ1Q2Gate(self.ctx, r1, r2, float(coeff))
        self._check()

    def ftQ2P(self, r: int) -> None:
        self._L.cvdvFtQ2P(self.ctx, r)
        self._check()

    def ftP2Q(self, r: int) -> None:
        self._L.cvdvFtP2Q(self.ctx, r)
        self._check()

    # -------------------------------------------------------------- readouts
    def synchronize(self) -> None:
        """(addition) run queued gates and wait for the GPU."""
        self._L.cvdvSynchronize(self.ctx)
        self._check()

    def getState(self) -> npt.NDArray[np.complex128]:
        re = np.zeros(self.total_size, dtype=np.float64)
        im = np.zeros(self.total_size, dtype=np.float64)
        self._L.cvdvGetState(self.ctx, _dptr(re), _dptr(im))
        self._check()
        return re + 1j * im

    def stateTensor(self) -> torch.Tensor:
        """(addition) zero-copy torch view of the live device state (complex128
        or complex64), valid until the next gate runs."""
        ptr = self._L.cvdvGetStateDevicePtr(self.ctx)
        self._check()
        if not ptr:
            raise CvdvError("state not initialised")
        typestr = "<c16" if PRECISIONS[self.precision] == 0 else "<c8"

        class _View:
            __cuda_array_interface__ = {"shape": (self.total_size,), "typestr": typestr,
                                        "data": (int(ptr), False), "version": 3,
                                        "stream": None}
        self._L.cvdvSynchronize(self.ctx)
        return torch.as_tensor(_View(), device="cuda")

    def getXGrid(self, r: int) -> npt.NDArray[np.float64]:
        N = self.register_dims[r]
        return (np.arange(N) - (N - 1) * 0.5) * self.grid_steps[r]

    def m(self, *regIdxs) -> "float | npt.NDArray[np.float64]":
        """No arguments: sum |psi|^2 (cvdvGetNorm).  Otherwise the joint marginal
        in C order over the listed registers (src/cudaCvdv.py:145-160)."""
        if len(regIdxs) == 1 and isinstance(regIdxs[0], (list, tuple)):
            regIdxs = tuple(regIdxs[0])
        if not regIdxs:
            v = float(self._L.cvdvGetNorm(self.ctx))
            self._check()
            return v
        regs = list(regIdxs)
        out = np.zeros(int(np.prod([self.register_dims[r] for r in regs])), dtype=np.float64)
        rc = (c_int * len(regs))(*regs)
        self._L.cvdvMeasureMultiple(self.ctx, rc, len(regs), _dptr(out))
        self._check()
        shape = tuple(self.register_dims[r] for r in regs)
        if len(shape) == 1:
            return out.reshape(shape)
        return out.reshape(shape[::-1]).T

    def mEach(self, regIdxs: List[int]) -> List[npt.NDArray[np.float64]]:
        """(addition) single-register marginals of several registers."""
        sizes = [self.register_dims[r] for r in regIdxs]
        out = np.zeros(sum(sizes), dtype=np.float64)
        rc = (c_int * len(regIdxs))(*regIdxs)
        self._L.cvdvMeasureEach(self.ctx, rc, len(regIdxs), _dptr(out))
        self._check()
        res, off = [], 0
        for s in sizes:
            res.append(out[off:off + s].copy())
            off += s
        return res

    def fidelityWith(self, other: "CudaCvdv") -> float:
        f = c_double(0.0)
        self._L.cvdvFidelityStatevectors(self.ctx, other.ctx, ctypes.byref(f))
        self._check()
        return float(f.value)

    def getFidelity(self, sep: SeparableState) -> float:
        sep.validate()
        ptrs = (ctypes.c_void_p * self.num_registers)(
            *[ctypes.c_void_p(a.data_ptr()) for a in sep.register_arrays])
        f = c_double(0.0)
        self._L.cvdvGetFidelity(self.ctx, ptrs, self.num_registers, ctypes.byref(f))
        self._check()
        return float(f.value)

    def getPhotonNumber(self, r: int) -> float:
        v = float(self._L.cvdvGetPhotonNumber(self.ctx, r))
        self._check()
        return v

    def _phase_space(self, fn, r: int) -> np.ndarray:
        N = self.register_dims[r]
        out = np.zeros(N * N, dtype=np.float64)
        fn(self.ctx, r, _dptr(out))
        self._check()
        return out.reshape(N, N)

    def getWigner(self, r: int, bound: Optional[float] = None) -> npt.NDArray[np.float64]:
        """Native N x N Wigner (row p, column x), clipped to |x|,|p| <= bound with
        dp = pi / (N dx) (src/cudaCvdv.py:186-197)."""
        W = self._phase_space(self._L.cvdvGetWigner, r)
        if bound is None:
            return W
        N, dx = self.register_dims[r], self.grid_steps[r]
        x = (np.arange(N) - (N - 1) / 2) * dx
        p = (np.arange(N) - N / 2) * (np.pi / (N * dx))
        return W[np.ix_(np.abs(p) <= bound, np.abs(x) <= bound)]

    def getHusimiQ(self, r: int, bound: Optional[float] = None) -> npt.NDArray[np.float64]:
        """Native N x N Husimi Q with dp = 2 pi / (N dx) (src/cudaCvdv.py:199-210)."""
        Q = self._phase_space(self._L.cvdvGetHusimiQ, r)
        if bound is None:
            return Q
        N, dx = self.register_dims[r], self.grid_steps[r]
        x = (np.arange(N) - (N - 1) / 2) * dx
        p = (np.arange(N) - N / 2) * (2 * np.pi / (N * dx))
        return Q[np.ix_(np.abs(p) <= bound, np.abs(x) <= bound)]

    def getHusimiQWigner(self, r: int) -> npt.NDArray[np.float64]:
        """(addition) cvdvGetHusimiQWigner: Gaussian-smoothed Wigner route."""
        return self._phase_space(self._L.cvdvGetHusimiQWigner, r)

    def plotWigner(self, r: int, bound: float = 5.0, cmap: str = "RdBu", figsize=(7, 6), show: bool = True) -> Tuple[Any, Any]:
        import matplotlib.pyplot as plt
        N, dx = self.register_dims[r], self.grid_steps[r]
        x = (np.arange(N) - (N - 1) / 2) * dx
        p = (np.arange(N) - N / 2) * (np.pi / (N * dx))
        W = self.getWigner(r, bound)
        fig, ax = plt.subplots(figsize=figsize)
        v = np.max(np.abs(W))
        im = ax.pcolormesh(x[np.abs(x) <= bound], p[np.abs(p) <= bound], W, cmap=cmap, vmin=-v, vmax=v, shading="auto")
        ax.set_xlabel(r"$q$")
        ax.set_ylabel(r"$p$")
        fig.colorbar(im, ax=ax)
        if show:
            plt.show()
        return fig, ax

    def plotHusimiQ(self, r: int, bound: float = 5.0, cmap: str = "viridis", figsize=(7, 6), show: bool = True) -> Tuple[Any, Any]:
        import matplotlib.pyplot as plt
        N, dx = self.register_dims[r], self.grid_steps[r]
        x = (np.arange(N) - (N - 1) / 2) * dx
        p = (np.arange(N) - N / 2) * (2 * np.pi / (N * dx))
        Q = self.getHusimiQ(r, bound)
        fig, ax = plt.subplots(figsize=figsize)
        im = ax.pcolormesh(x[np.abs(x) <= bound], p[np.abs(p) <= bound], Q, cmap=cmap, shading="auto")
        ax.set_xlabel(r"$q$")
        ax.set_ylabel(r"$p$")
        fig.colorbar(im, ax=ax)
        if show:
            plt.show()
        return fig, ax
