"""CPU restatement of CUDA-CVDV's dense state-vector path (numpy, complex128).

TEST INFRASTRUCTURE ONLY.  This module is the parity checker for the CUDA
library under ``cuda-cvdv_b200/``.  Only ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import
it, and only as the thing results are checked against (or, in ``bench.py``, as
the timed CPU implementation).  The product path never imports it.

Parity is pinned: ``tests/golden/make_golden.py`` ran the reference's own
``TorchCvdv`` (complex128, CPU) and stored its outputs under ``tests/golden/``;
``tests/test_oracle_golden.py`` checks this module against those fixtures and
against the reference tests' known answers (closed-form Wigner/Husimi,
numpy ftQ2P restatement, identities).

Conventions followed (all citations are paths inside the reference project):

* register layout: register 0 is the most significant, the last register
  varies fastest; ``flw_r = sum(q_s for s > r)``; local index
  ``j_r = (i >> flw_r) & (N_r - 1)`` (``src/cuda/context.cu:26-38``,
  ``src/cuda/kernels/utils.cuh:34-37``);
* qubit k of register r lives at global bit ``flw_r + q_r - 1 - k``
  (``src/cuda/kernels/utils.cuh:74-84``);
* grid ``x_j = (j - (N-1)/2) dx``, ``dx = sqrt(2 pi / N)``
  (``src/cuda/kernels/utils.cuh:5-7``, ``src/cuda/context.cu:30-31``);
* every gate is decomposed exactly as ``src/cuda/gates.cu`` does, with the
  same thresholds, rounding functions and global-phase choices.
"""

from __future__ import annotations

import math
from typing import List, Sequence

import numpy as np

try:  # multi-threaded FFT when scipy is present (CPU baseline speed only)
    import scipy.fft as _sfft

    def _fft(a, axis, workers):
        return _sfft.fft(a, axis=axis, workers=workers)

    def _ifft_unnorm(a, axis, workers):
        return _sfft.ifft(a, axis=axis, norm="forward", workers=workers)

except ImportError:  # pragma: no cover
    def _fft(a, axis, workers):
        return np.fft.fft(a, axis=axis)

    def _ifft_unnorm(a, axis, workers):
        return np.fft.ifft(a, axis=axis, norm="forward")


PI = 3.14159265358979323846
SQRT2 = 1.41421356237309504880

_POOLS: dict = {}


def _pool(workers: int):
    """Shared thread pool for the elementwise passes (numpy releases the GIL
    inside its loops, so chunks of one multiply run on separate cores)."""
    if workers <= 1:
        return None
    if workers not in _POOLS:
        from concurrent.futures import ThreadPoolExecutor
        _POOLS[workers] = ThreadPoolExecutor(max_workers=workers)
    return _POOLS[workers]


def _ranges(n: int, parts: int):
    step = -(-n // parts)
    return [(a, min(a + step, n)) for a in range(0, n, step)]


# states smaller than this stay on the single-threaded numpy path
_THREAD_MIN = 1 << 20


def c_round(x: float) -> float:
    """C ``round()``: halves away from zero (used by ``gates.cu:470,514``)."""
    return math.copysign(math.floor(abs(x) + 0.5), x)


class OracleCvdv:
    """numpy mirror of one ``CVDVContext`` (``src/cuda/types.h:54-77``)."""

    def __init__(self, qubits: Sequence[int], workers: int = 1) -> None:
        self.q: List[int] = [int(v) for v in qubits]
        self.R = len(self.q)
        self.dims = [1 << v for v in self.q]
        self.n = sum(self.q)
        self.size = 1 << self.n
        # context.cu:33-38
        self.flw = [sum(self.q[r + 1:]) for r in range(self.R)]
        # context.cu:30-31
        self.dx = [math.sqrt(2.0 * PI / d) for d in self.dims]
        self.state: np.ndarray | None = None
        self.workers = workers

    # ------------------------------------------------------------ helpers
    def _t(self) -> np.ndarray:
        """State viewed as an R-dimensional array indexed by local indices."""
        return self.state.reshape(self.dims)

    def grid(self, r: int) -> np.ndarray:
        """``gridX`` of ``src/cuda/kernels/utils.cuh:5-7`` for every local index."""
        N = self.dims[r]
        j = np.arange(N, dtype=np.float64)
        return (j - (N - 1) * 0.5) * self.dx[r]

    def _bcast(self, vec: np.ndarray, axis: int) -> np.ndarray:
        shape = [1] * self.R
        shape[axis] = -1
        return vec.reshape(shape)

    def _mul(self, fac) -> None:
        """``state *= fac`` with ``fac`` broadcastable to the register-indexed
        shape.  With ``workers > 1`` the state is cut into slabs along its
        leading registers and the slabs are multiplied in place on a thread
        pool; elementwise, so every amplitude gets the same product."""
        fac = np.asarray(fac)
        fac = fac.reshape((1,) * (self.R - fac.ndim) + fac.shape)
        pool = _pool(self.workers)
        if pool is None or self.size < _THREAD_MIN:
            self.state = (self._t() * fac).reshape(-1)
            return
        s, P = 0, 1
        while s < self.R and P < 16 * self.workers:
            P *= self.dims[s]
            s += 1
        st = np.ascontiguousarray(self.state)
        tv = st.reshape((P,) + tuple(self.dims[s:]))
        fv = np.broadcast_to(fac, tuple(self.dims[:s]) + fac.shape[s:]).reshape((P,) + fac.shape[s:])

        def run(ab):
            a, b = ab
            np.multiply(tv[a:b], fv[a:b], out=tv[a:b])

        list(pool.map(run, _ranges(P, 4 * self.workers)))
        self.state = st

    def _ctrl_sign(self, ctrl_reg: int, ctrl_qubit: int) -> np.ndarray:
        """+1 where the control qubit is 0, -1 where it is 1 (``gates.cuh:31-37``)."""
        Nc = self.dims[ctrl_reg]
        mask = 1 << (self.q[ctrl_reg] - 1 - ctrl_qubit)
        jc = np.arange(Nc)
        return np.where(jc & mask, -1.0, 1.0)

    def _apply_phase_2d(self, phase_fn, reg_a: int, reg_b: int) -> None:
        """Multiply by exp(i*phase(j_a, j_b)); handles reg_a == reg_b."""
        if reg_a == reg_b:
            ph = phase_fn(np.arange(self.dims[reg_a]), np.arange(self.dims[reg_a]), diag=True)
            self._mul(self._bcast(np.exp(1j * ph), reg_a))
            return
        ja = np.arange(self.dims[reg_a])[:, None]
        jb = np.arange(self.dims[reg_b])[None, :]
        ph = phase_fn(ja, jb, diag=False)
        fac = np.exp(1j * ph)
        shape = [1] * self.R
        shape[reg_a] = self.dims[reg_a]
        shape[reg_b] = self.dims[reg_b]
        if reg_a > reg_b:
            fac = fac.T
        self._mul(fac.reshape(shape))

    # ------------------------------------------------------------ init / io
    def init_from_separable(self, arrays: Sequence[np.ndarray]) -> None:
        """Tensor product, last register fastest, NOT normalised
        (``src/cuda/context.cu:75-115``)."""
        assert len(arrays) == self.R
        st = np.ones(1, dtype=np.complex128)
        for r in range(self.R):
            a = np.asarray(arrays[r], dtype=np.complex128).reshape(-1)
            assert a.size == self.dims[r]
            st = np.multiply.outer(st, a).reshape(-1)
        self.state = st

    def set_state(self, arr) -> None:
        """``cvdvSetStateFromDevicePtr`` (``src/cuda/context.cu:131-137``)."""
        a = np.asarray(arr, dtype=np.complex128).reshape(-1)
        assert a.size == self.size
        self.state = a.copy()

    def get_state(self) -> np.ndarray:
        return self.state.copy()

    # ------------------------------------------------------------ diagonal kernels
    def phase_x(self, r: int, c: float) -> None:
        """``kernelPhaseX`` (``gates.cuh:5-16``): psi *= exp(i c x)."""
        ph = c * self.grid(r)
        self._mul(self._bcast(np.exp(1j * ph), r))

    def cphase_x(self, t: int, cr: int, cq: int, c: float) -> None:
        """``kernelCPhaseX`` (``gates.cuh:20-38``): exp(i c Z x)."""
        x = self.grid(t)
        sg = self._ctrl_sign(cr, cq)
        self._apply_phase_2d(
            lambda jt, jc, diag: (sg[jc] * (c * x[jt])) if not diag else sg[jt] * (c * x[jt]),
            t, cr)

    def phase_x2(self, r: int, tcoef: float) -> None:
        """``kernelPhaseX2`` (``gates.cuh:184-196``): exp(i t x^2)."""
        x = self.grid(r)
        self._mul(self._bcast(np.exp(1j * (tcoef * x * x)), r))

    def cphase_x2(self, t: int, cr: int, cq: int, tcoef: float) -> None:
        """``kernelCPhaseX2`` (``gates.cuh:42-60``): exp(i t Z x^2)."""
        x = self.grid(t)
        sg = self._ctrl_sign(cr, cq)
        self._apply_phase_2d(
            lambda jt, jc, diag: (sg[jc] * (tcoef * x[jt] * x[jt])) if not diag
            else sg[jt] * (tcoef * x[jt] * x[jt]),
            t, cr)

    def phase_x3(self, r: int, c: float) -> None:
        """``kernelPhaseX3`` (``gates.cuh:198-209``): exp(i c x^3)."""
        x = self.grid(r)
        self._mul(self._bcast(np.exp(1j * (c * x * x * x)), r))

    def phase_xx(self, r1: int, r2: int, c: float) -> None:
        """``kernelPhaseXX`` (``gates.cuh:213-231``): exp(i c x1 x2)."""
        x1, x2 = self.grid(r1), self.grid(r2)
        self._apply_phase_2d(lambda a, b, diag: c * x1[a] * x2[b], r1, r2)

    def cphase_xx(self, r1: int, r2: int, cr: int, cq: int, c: float) -> None:
        """``kernelCPhaseXX`` (``gates.cuh:235-259``): exp(i c Z x1 x2), flat form."""
        idx = np.arange(self.size, dtype=np.int64)
        j1 = (idx >> self.flw[r1]) & (self.dims[r1] - 1)
        j2 = (idx >> self.flw[r2]) & (self.dims[r2] - 1)
        bit = (idx >> (self.flw[cr] + self.q[cr] - 1 - cq)) & 1
        ph = c * self.grid(r1)[j1] * self.grid(r2)[j2]
        ph = np.where(bit == 1, -ph, ph)
        self.state = self.state * np.exp(1j * ph)

    def global_scalar(self, s: float) -> None:
        """``kernelGlobalScalar`` (``gates.cuh:262-268``)."""
        self._mul(np.float64(s))

    def global_phase(self, phi: float) -> None:
        """``kernelGlobalPhase`` (``gates.cuh:271-275``)."""
        self._mul(np.exp(1j * phi))

    # ------------------------------------------------------------ basis change
    def ft_q2p(self, r: int) -> None:
        """``cvdvFtQ2P`` (``gates.cu:19-67``)."""
        N = self.dims[r]
        coeff = PI * (N - 1.0) / (N * self.dx[r])
        self.phase_x(r, coeff)
        self.state = _fft(self._t(), r, self.workers).reshape(-1)
        self.phase_x(r, coeff)
        self.global_scalar(1.0 / math.sqrt(float(N)))
        self.global_phase(PI * float(N - 1) * float(N - 1) / (2.0 * float(N)))

    def ft_p2q(self, r: int) -> None:
        """``cvdvFtP2Q`` (``gates.cu:69-122``); CUFFT_INVERSE is unnormalised."""
        N = self.dims[r]
        coeff = -PI * (N - 1.0) / (N * self.dx[r])
        self.phase_x(r, coeff)
        self.state = _ifft_unnorm(self._t(), r, self.workers).reshape(-1)
        self.phase_x(r, coeff)
        self.global_scalar(1.0 / math.sqrt(float(N)))
        self.global_phase(-PI * float(N - 1) * float(N - 1) / (2.0 * float(N)))

    # ------------------------------------------------------------ qubit gates
    def _pair(self, r: int, k: int, m00, m01, m10, m11) -> None:
        """2x2 update on the pairs differing in one bit (``utils.cuh:79-84``)."""
        b = self.flw[r] + self.q[r] - 1 - k
        pool = _pool(self.workers)
        if pool is not None and self.size >= _THREAD_MIN:
            self._pair_threaded(pool, b, m00, m01, m10, m11)
            return
        v = self.state.reshape(-1, 2, 1 << b)
        a0 = v[:, 0, :].copy()
        a1 = v[:, 1, :].copy()
        out = np.empty_like(v)
        out[:, 0, :] = m00 * a0 + m01 * a1
        out[:, 1, :] = m10 * a0 + m11 * a1
        self.state = out.reshape(-1)

    def _pair_threaded(self, pool, b: int, m00, m01, m10, m11) -> None:
        """``_pair`` in place, slabs of pairs on the thread pool."""
        st = np.ascontiguousarray(self.state)
        v = st.reshape(-1, 2, 1 << b)
        A, B = v.shape[0], v.shape[2]
        parts = 4 * self.workers

        def run(ab):
            a, e = ab
            sl = (slice(a, e), slice(None)) if A >= parts else (slice(None), slice(a, e))
            a0 = v[sl[0], 0, sl[1]].copy()
            a1 = v[sl[0], 1, sl[1]]
            v[sl[0], 0, sl[1]] = m00 * a0 + m01 * a1
            v[sl[0], 1, sl[1]] = m10 * a0 + m11 * a1

        list(pool.map(run, _ranges(A if A >= parts else B, parts)))
        self.state = st

    def pauli_rotation(self, r: int, k: int, axis: int, theta: float) -> None:
        """``kernelPauliRotation`` (``gates.cuh:63-92``)."""
        c, s = math.cos(theta / 2.0), math.sin(theta / 2.0)
        if axis == 0:
            self._pair(r, k, c, -1j * s, -1j * s, c)
        elif axis == 1:
            self._pair(r, k, c, -s, s, c)
        else:
            self._pair(r, k, complex(c, -s), 0.0, 0.0, complex(c, s))

    def hadamard(self, r: int, k: int) -> None:
        """``kernelHadamard`` (``gates.cuh:95-109``)."""
        h = 1.0 / SQRT2
        self._pair(r, k, h, h, h, -h)

    # ------------------------------------------------------------ permutations
    def parity(self, r: int) -> None:
        """``kernelParity`` (``gates.cuh:113-131``): j -> N-1-j."""
        self.state = np.flip(self._t(), axis=r).reshape(-1).copy()

    def cparity(self, t: int, cr: int, cq: int) -> None:
        """``kernelConditionalParity`` (``gates.cuh:134-158``), flat form so that
        a control inside the target register behaves exactly as the kernel."""
        idx = np.arange(self.size, dtype=np.int64)
        bit = (idx >> (self.flw[cr] + self.q[cr] - 1 - cq)) & 1
        N = self.dims[t]
        loc = (idx >> self.flw[t]) & (N - 1)
        flipped = (N - 1) - loc
        act = (bit == 1) & (loc < flipped)
        src = idx[act]
        dst = src + (flipped[act] - loc[act]) * (1 << self.flw[t])
        out = self.state.copy()
        out[src] = self.state[dst]
        out[dst] = self.state[src]
        self.state = out

    def swap(self, r1: int, r2: int) -> None:
        """``kernelSwapRegisters`` (``gates.cuh:161-182``); no-op on mismatch
        (``gates.cu:271-279``)."""
        if self.q[r1] != self.q[r2] or r1 == r2:
            return
        self.state = np.swapaxes(self._t(), r1, r2).reshape(-1).copy()

    # ------------------------------------------------------------ composite gates
    def displacement(self, r: int, re: float, im: float) -> None:
        """``cvdvDisplacement`` (``gates.cu:124-161``); global phase dropped."""
        if abs(im) > 1e-12:
            self.phase_x(r, SQRT2 * im)
        if abs(re) > 1e-12:
            self.ft_q2p(r)
            self.phase_x(r, -SQRT2 * re)
            self.ft_p2q(r)

    def cond_displacement(self, t: int, cr: int, cq: int, re: float, im: float) -> None:
        """``cvdvConditionalDisplacement`` (``gates.cu:163-204``)."""
        if abs(im) > 1e-12:
            self.cphase_x(t, cr, cq, SQRT2 * im)
        if abs(re) > 1e-12:
            self.ft_q2p(t)
            self.cphase_x(t, cr, cq, -SQRT2 * re)
            self.ft_p2q(t)

    def _rotation_small(self, r: int, theta: float) -> None:
        """``cvdvRotationSmall`` (``gates.cu:572-584``)."""
        if abs(theta) < 1e-15:
            return
        th = math.tan(theta / 2.0)
        st = math.sin(theta)
        self.phase_x2(r, -0.5 * th)
        self.ft_q2p(r)
        self.phase_x2(r, -0.5 * st)
        self.ft_p2q(r)
        self.phase_x2(r, -0.5 * th)

    def rotation(self, r: int, theta: float) -> None:
        """``cvdvRotation`` (``gates.cu:316-348``); ``rint`` = half to even."""
        theta0 = float(np.rint(theta / (PI / 2.0))) * (PI / 2.0)
        rem = theta - theta0
        qt = int(np.rint(theta0 / (PI / 2.0)))
        qt = ((qt % 4) + 4) % 4
        if qt == 1:
            self.ft_q2p(r)
        elif qt == 2:
            self.parity(r)
        elif qt == 3:
            self.ft_p2q(r)
        self._rotation_small(r, rem)

    def _cond_rotation_small(self, t: int, cr: int, cq: int, theta: float) -> None:
        """``cvdvConditionalRotationSmall`` (``gates.cu:598-611``)."""
        if abs(theta) < 1e-15:
            return
        th = math.tan(theta / 2.0)
        st = math.sin(theta)
        self.cphase_x2(t, cr, cq, -0.5 * th)
        self.ft_q2p(t)
        self.cphase_x2(t, cr, cq, -0.5 * st)
        self.ft_p2q(t)
        self.cphase_x2(t, cr, cq, -0.5 * th)

    def cond_rotation(self, t: int, cr: int, cq: int, theta: float) -> None:
        """``cvdvConditionalRotation`` (``gates.cu:350-392``)."""
        theta0 = float(np.rint(theta / (PI / 2.0))) * (PI / 2.0)
        rem = theta - theta0
        qt = int(np.rint(theta0 / (PI / 2.0)))
        qt = ((qt % 4) + 4) % 4
        if qt == 1:
            self.ft_q2p(t)
            self.cparity(t, cr, cq)
            self.pauli_rotation(cr, cq, 2, PI / 2)
        elif qt == 2:
            self.parity(t)
            self.pauli_rotation(cr, cq, 2, PI)
        elif qt == 3:
            self.ft_p2q(t)
            self.cparity(t, cr, cq)
            self.pauli_rotation(cr, cq, 2, -PI / 2)
        self._cond_rotation_small(t, cr, cq, rem)

    def squeeze(self, r: int, rr: float) -> None:
        """``cvdvSqueeze`` (``gates.cu:394-421``)."""
        a = math.exp(0.5 * rr)
        b = math.exp(-0.5 * rr)
        s = math.sqrt(abs(math.exp(rr) - 1.0))
        sg = 1.0 if rr >= 0 else -1.0
        self.ft_q2p(r)
        self.phase_x2(r, -0.5 * a * s)
        self.ft_p2q(r)
        self.phase_x2(r, 0.5 * b * s * sg)
        self.ft_q2p(r)
        self.phase_x2(r, 0.5 * b * s)
        self.ft_p2q(r)
        self.phase_x2(r, -0.5 * a * s * sg)

    def cond_squeeze(self, t: int, cr: int, cq: int, rr: float) -> None:
        """``cvdvConditionalSqueeze`` (``gates.cu:423-459``)."""
        ch = math.cosh(rr)
        sh = math.sinh(rr)
        s = math.sqrt(2.0 * abs(math.sinh(0.5 * rr)))
        self.phase_x2(t, 0.5 * s * ch)
        self.cphase_x2(t, cr, cq, -0.5 * s * sh)
        self.ft_q2p(t)
        self.phase_x2(t, 0.5 * (ch - 1) / s)
        self.cphase_x2(t, cr, cq, 0.5 * sh / s)
        self.ft_p2q(t)
        self.phase_x2(t, -0.5 * s)
        self.ft_q2p(t)
        self.phase_x2(t, 0.5 * (ch - 1) / s)
        self.cphase_x2(t, cr, cq, -0.5 * sh / s)
        self.ft_p2q(t)

    def _bs_small(self, r1: int, r2: int, theta: float) -> None:
        """``cvdvBeamSplitterSmall`` (``gates.cu:614-636``)."""
        if abs(theta) < 1e-15:
            return
        cq = -math.tan(0.25 * theta)
        cp = -math.sin(0.5 * theta)
        self.phase_xx(r1, r2, cq)
        self.ft_q2p(r1)
        self.ft_q2p(r2)
        self.phase_xx(r1, r2, cp)
        self.ft_p2q(r1)
        self.ft_p2q(r2)
        self.phase_xx(r1, r2, cq)

    def beam_splitter(self, r1: int, r2: int, theta: float) -> None:
        """``cvdvBeamSplitter`` (``gates.cu:461-502``); ``round`` = half away."""
        theta0 = c_round(theta / PI) * PI
        rem = theta - theta0
        ht = int(c_round(theta0 / PI))
        ht = ((ht % 4) + 4) % 4
        if ht == 1:
            self.ft_q2p(r1)
            self.ft_q2p(r2)
            self.swap(r1, r2)
        elif ht == 2:
            self.parity(r1)
            self.parity(r2)
        elif ht == 3:
            self.ft_p2q(r1)
            self.ft_p2q(r2)
            self.swap(r1, r2)
        self._bs_small(r1, r2, rem)

    def _cbs_small(self, r1: int, r2: int, cr: int, cq: int, theta: float) -> None:
        """``cvdvConditionalBeamSplitterSmall`` (``gates.cu:640-666``)."""
        if abs(theta) < 1e-15:
            return
        cqq = -math.tan(0.25 * theta)
        cpp = -math.sin(0.5 * theta)
        self.cphase_xx(r1, r2, cr, cq, cqq)
        self.ft_q2p(r1)
        self.ft_q2p(r2)
        self.cphase_xx(r1, r2, cr, cq, cpp)
        self.ft_p2q(r1)
        self.ft_p2q(r2)
        self.cphase_xx(r1, r2, cr, cq, cqq)

    def cond_beam_splitter(self, r1: int, r2: int, cr: int, cq: int, theta: float) -> None:
        """``cvdvConditionalBeamSplitter`` (``gates.cu:504-547``)."""
        theta0 = c_round(theta / PI) * PI
        rem = theta - theta0
        ht = int(c_round(theta0 / PI))
        ht = ((ht % 4) + 4) % 4
        if ht == 1:
            self.ft_q2p(r1)
            self.ft_q2p(r2)
            self.cparity(r1, cr, cq)
            self.cparity(r2, cr, cq)
            self.swap(r1, r2)
        elif ht == 2:
            self.parity(r1)
            self.parity(r2)
        elif ht == 3:
            self.ft_p2q(r1)
            self.ft_p2q(r2)
            self.cparity(r1, cr, cq)
            self.cparity(r2, cr, cq)
            self.swap(r1, r2)
        self._cbs_small(r1, r2, cr, cq, rem)

    def q1q2(self, r1: int, r2: int, c: float) -> None:
        """``cvdvQ1Q2Gate`` (``gates.cu:549-565``); same register is rejected."""
        if r1 == r2:
            return
        self.phase_xx(r1, r2, c)

    # ------------------------------------------------------------ readouts
    def measure_multiple(self, regs: Sequence[int]) -> np.ndarray:
        """``cvdvMeasureMultiple`` (``measure.cu:65-123``): flat output, first
        selected register fastest (column-major)."""
        regs = list(regs)
        ext = [self.dims[r] for r in regs]
        strides = [1]
        for e in ext[:-1]:
            strides.append(strides[-1] * e)
        out_size = int(np.prod(ext))
        p = np.abs(self.state) ** 2
        idx = np.arange(self.size, dtype=np.int64)
        oi = np.zeros(self.size, dtype=np.int64)
        for r, st in zip(regs, strides):
            oi += ((idx >> self.flw[r]) & (self.dims[r] - 1)) * st
        return np.bincount(oi, weights=p, minlength=out_size)

    def m(self, *regs):
        """``CudaCvdv.m`` (``src/cudaCvdv.py:145-160``): no args -> sum |psi|^2
        (``measure.cu:276-300``), else C-order marginal over ``regs``."""
        if len(regs) == 1 and isinstance(regs[0], (list, tuple)):
            regs = tuple(regs[0])
        if not regs:
            return float(np.sum(np.abs(self.state) ** 2))
        out = self.measure_multiple(regs)
        shape = tuple(self.dims[r] for r in regs)
        if len(shape) == 1:
            return out.reshape(shape)
        return out.reshape(shape[::-1]).T

    def get_norm(self) -> float:
        return float(np.sum(np.abs(self.state) ** 2))

    def get_fidelity(self, arrays: Sequence[np.ndarray]) -> float:
        """``cvdvGetFidelity`` (``measure.cu:302-318`` via ``measure.cuh:182-223``):
        |sum conj(psi) * prod_r phi_r|^2."""
        ref = np.ones(1, dtype=np.complex128)
        for a in arrays:
            ref = np.multiply.outer(ref, np.asarray(a, dtype=np.complex128).reshape(-1)).reshape(-1)
        ip = np.sum(np.conj(self.state) * ref)
        return float(ip.real ** 2 + ip.imag ** 2)

    def expect_x2(self, r: int) -> float:
        """``kernelExpectX2`` (``measure.cuh:158-178``)."""
        x = self.grid(r)
        return float(np.sum(np.abs(self._t()) ** 2 * self._bcast(x * x, r)))

    def photon_number(self, r: int) -> float:
        """``cvdvGetPhotonNumber`` (``measure.cu:320-331``): (<q^2>+<p^2>-1)/2."""
        q2 = self.expect_x2(r)
        self.ft_q2p(r)
        p2 = self.expect_x2(r)
        self.ft_p2q(r)
        return (q2 + p2 - 1.0) / 2.0

    def fidelity_with(self, other: "OracleCvdv") -> float:
        """``cvdvFidelityStatevectors`` (``measure.cu:333-366``)."""
        ip = np.sum(np.conj(self.state) * other.state)
        return float(ip.real ** 2 + ip.imag ** 2)

    # -------------------------------------------------------- phase space
    def target_slices(self, r: int) -> np.ndarray:
        """[slices, N] with the slice index ordered as ``kernelExtractChunkPsi``
        (``bosonic.cuh:93-106``): low bits below the register, then high bits."""
        N = self.dims[r]
        t = self.state.reshape(1 << (self.n - self.q[r] - self.flw[r]), N, 1 << self.flw[r])
        return np.transpose(t, (0, 2, 1)).reshape(-1, N)

    def wigner_g(self, r: int) -> np.ndarray:
        """``kernelBuildWignerRow`` (``bosonic.cuh:7-36``):
        G[i,k] = sum_o conj(psi_o[i+kd]) psi_o[i-kd], kd = k - (N-1)//2."""
        N = self.dims[r]
        S = self.target_slices(r)
        rho = S.T @ np.conj(S)  # rho[a, b] = sum_o psi_o[a] conj(psi_o[b])
        i = np.arange(N)[:, None]
        kd = np.arange(N)[None, :] - (N - 1) // 2
        ip, im = i + kd, i - kd
        valid = (ip >= 0) & (ip < N) & (im >= 0) & (im < N)
        G = np.where(valid, rho[np.clip(im, 0, N - 1), np.clip(ip, 0, N - 1)], 0.0)
        return G

    def wigner(self, r: int) -> np.ndarray:
        """``cvdvGetWigner`` (``bosonic.cu:103-132``) + ``kernelFinalizeWigner``
        (``bosonic.cuh:39-52``): W[jc, i] on the native N x N grid."""
        N = self.dims[r]
        dx = self.dx[r]
        H = np.fft.ifft(self.wigner_g(r), axis=1) * N  # CUFFT_INVERSE, unnormalised
        jc = np.arange(N)
        kf = (jc + N // 2) % N
        pj = (jc - N / 2.0) * PI / (float(N) * dx)
        ph = -pj * (N - 1) * dx
        G = H[:, kf].T  # [jc, i]
        return (G.real * np.cos(ph)[:, None] - G.imag * np.sin(ph)[:, None]) * dx / PI

    def husimi_g(self, r: int) -> np.ndarray:
        """``kernelComputeHusimiG`` (``bosonic.cuh:82-89``)."""
        N = self.dims[r]
        dx = self.dx[r]
        k = np.arange(N)
        ks = np.where(k <= N // 2, k, k - N)
        pe = 2.0 * math.pi * ks / (float(N) * dx)
        return (math.pi ** 0.25) * math.sqrt(2.0 / dx) * np.exp(-0.5 * pe * pe)

    def husimi(self, r: int) -> np.ndarray:
        """``husimiFromOverlap`` (``bosonic.cu:10-61``) with kernels
        ``bosonic.cuh:93-147``: Q[jc, q] = sum_s |IFFT_k(Psi_s[(m+k)%N] G[k])[q]|^2
        / (pi N^2) at m = (jc + N/2) % N."""
        N = self.dims[r]
        S = self.target_slices(r)
        Psi = np.fft.fft(S, axis=1)
        G = self.husimi_g(r)
        m = np.arange(N)[:, None]
        k = np.arange(N)[None, :]
        idx = (m + k) & (N - 1)
        acc = np.zeros((N, N))
        for s in range(S.shape[0]):
            A = Psi[s][idx] * G[None, :]
            H = np.fft.ifft(A, axis=1) * N
            acc += H.real ** 2 + H.imag ** 2
        jc = np.arange(N)
        return acc[(jc + N // 2) % N, :] / (PI * float(N) * float(N))

    def husimi_wigner(self, r: int) -> np.ndarray:
        """``husimiFromWignerFft2`` (``bosonic.cu:63-101``) with kernels
        ``bosonic.cuh:56-70,158-186``: Gaussian smoothing of W by 2-D FFT."""
        N = self.dims[r]
        dx = self.dx[r]
        W = self.wigner(r).astype(np.complex128)
        F = np.fft.fft2(W)
        p = np.arange(N)[:, None]
        q = np.arange(N)[None, :]
        kq = np.where(q <= N // 2, q, q - N)
        kp = np.where(p <= N // 2, p, p - N)
        Lq = float(N) * dx
        dp = PI / (float(N) * dx)
        Lp = float(N) * dp
        wq = 2.0 * PI * kq / Lq
        wp = 2.0 * PI * kp / Lp
        F = F * np.exp(-0.25 * (wq * wq + wp * wp))
        out = np.fft.ifft2(F).real  # = unnormalised inverse / N^2
        return np.maximum(out, 0.0)


class OracleSim(OracleCvdv):
    """The oracle behind the ``CudaCvdv`` method names (``src/cudaCvdv.py:77-252``),
    so one gate list drives both the CUDA library and the checker."""

    def initStateVector(self, sep) -> None:
        self.init_from_separable([np.asarray(a.cpu().numpy()) for a in sep.register_arrays])

    def initFromArray(self, arr) -> None:
        self.set_state(np.asarray(arr))

    def getState(self):
        return self.get_state()

    def d(self, r, beta):
        beta = complex(beta)
        self.displacement(r, beta.real, beta.imag)

    def cd(self, t, c, q, alpha):
        alpha = complex(alpha)
        self.cond_displacement(t, c, q, alpha.real, alpha.imag)

    def cr(self, t, c, q, theta):
        self.cond_rotation(t, c, q, theta)

    def x(self, r, k):
        self.pauli_rotation(r, k, 0, PI)

    def y(self, r, k):
        self.pauli_rotation(r, k, 1, PI)

    def z(self, r, k):
        self.pauli_rotation(r, k, 2, PI)

    def rx(self, r, k, t):
        self.pauli_rotation(r, k, 0, t)

    def ry(self, r, k, t):
        self.pauli_rotation(r, k, 1, t)

    def rz(self, r, k, t):
        self.pauli_rotation(r, k, 2, t)

    def h(self, r, k):
        self.hadamard(r, k)

    def p(self, r):
        self.parity(r)

    def cp(self, t, c, q):
        self.cparity(t, c, q)

    def sheer(self, r, t):
        self.phase_x2(r, t)

    def phaseCubic(self, r, t):
        self.phase_x3(r, t)

    def r(self, r, theta):
        self.rotation(r, theta)

    def s(self, r, rr):
        self.squeeze(r, rr)

    def cs(self, t, c, q, rr):
        self.cond_squeeze(t, c, q, rr)

    def bs(self, a, b, theta):
        self.beam_splitter(a, b, theta)

    def cbs(self, a, b, c, q, theta):
        self.cond_beam_splitter(a, b, c, q, theta)

    def ftQ2P(self, r):
        self.ft_q2p(r)

    def ftP2Q(self, r):
        self.ft_p2q(r)

    def getWigner(self, r, bound=None):
        W = self.wigner(r)
        if bound is None:
            return W
        N, dx = self.dims[r], self.dx[r]
        x = (np.arange(N) - (N - 1) / 2) * dx
        p = (np.arange(N) - N / 2) * (PI / (N * dx))
        return W[np.ix_(np.abs(p) <= bound, np.abs(x) <= bound)]

    def getHusimiQ(self, r, bound=None):
        Q = self.husimi(r)
        if bound is None:
            return Q
        N, dx = self.dims[r], self.dx[r]
        x = (np.arange(N) - (N - 1) / 2) * dx
        p = (np.arange(N) - N / 2) * (2 * PI / (N * dx))
        return Q[np.ix_(np.abs(p) <= bound, np.abs(x) <= bound)]

    def getPhotonNumber(self, r):
        return self.photon_number(r)

    def getFidelity(self, sep):
        return self.get_fidelity([np.asarray(a.cpu().numpy()) for a in sep.register_arrays])

    def fidelityWith(self, other):
        return self.fidelity_with(other)
