"""Accuracy readouts of a state or a phase-space grid against a reference one.

``compare_states`` streams two device states (any mix of complex128 and
complex64) in chunks, accumulating in complex128 on the GPU:

  infidelity    1 - |<ref|psi>|^2 / (<ref|ref> <psi|psi>)
  max_abs_err   max_i |psi_i - ref_i|
  rel_l2        ||psi - ref|| / ||ref||

``wigner_grid`` resamples a native N x N Wigner array (row p, column x, the
layout of ``CudaCvdv.getWigner``) onto an n x n grid over [-bound, bound]^2
(optionally shifted to a centre, e.g. ``wigner_mean``) by bilinear
interpolation in FP64 on the native lattice
  x_j = (j - (N-1)/2) dx,  p_k = (k - N/2) pi / (N dx),  dx = sqrt(2 pi / N)
(src/cudaCvdv.py:186-197 gives the native lattice).  The same deterministic
map applied to two native arrays gives grids whose difference is bounded by the
native difference, so grid errors are comparable across precisions.
"""

from __future__ import annotations

import math
from typing import Dict

import numpy as np
import torch


def compare_states(ref: torch.Tensor, psi: torch.Tensor, chunk: int = 1 << 24) -> Dict[str, float]:
    if ref.numel() != psi.numel():
        raise ValueError("states of different sizes")
    inner = torch.zeros((), dtype=torch.complex128, device=ref.device)
    n_ref = torch.zeros((), dtype=torch.float64, device=ref.device)
    n_psi = torch.zeros_like(n_ref)
    err2 = torch.zeros_like(n_ref)
    emax = torch.zeros_like(n_ref)
    for s in range(0, ref.numel(), chunk):
        a = ref[s:s + chunk].to(torch.complex128)
        b = psi[s:s + chunk].to(torch.complex128)
        inner += torch.sum(a.conj() * b)
        n_ref += torch.sum(a.real * a.real + a.imag * a.imag)
        n_psi += torch.sum(b.real * b.real + b.imag * b.imag)
        d = torch.abs(b - a)
        err2 += torch.sum(d * d)
        emax = torch.maximum(emax, d.max())
    ov = float(torch.abs(inner) ** 2 / (n_ref * n_psi))
    return {"infidelity": max(0.0, 1.0 - ov), "infidelity_raw": 1.0 - ov,
            "max_abs_err": float(emax), "rel_l2": math.sqrt(float(err2 / n_ref))}


def native_axes(N: int):
    dx = math.sqrt(2.0 * math.pi / N)
    x = (np.arange(N) - (N - 1) / 2.0) * dx
    p = (np.arange(N) - N / 2.0) * (math.pi / (N * dx))
    return x, p


def _weights(axis: np.ndarray, pts: np.ndarray):
    step = axis[1] - axis[0]
    u = (pts - axis[0]) / step
    i0 = np.clip(np.floor(u).astype(np.int64), 0, len(axis) - 2)
    f = u - i0
    return i0, f


def wigner_mean(W: np.ndarray):
    """(<x>, <p>) of a native Wigner array: sum x W / sum W and sum p W / sum W."""
    N = W.shape[0]
    x, p = native_axes(N)
    W = np.asarray(W, dtype=np.float64)
    tot = W.sum()
    return float((W.sum(axis=0) * x).sum() / tot), float((W.sum(axis=1) * p).sum() / tot)


def wigner_grid(W: np.ndarray, n: int = 256, bound: float = 6.0, center=(0.0, 0.0)) -> np.ndarray:
    """Bilinear FP64 resampling of a native Wigner array onto n x n points
    center + linspace(-bound, bound, n) in p (rows) and x (columns); center is
    (x0, p0)."""
    N = W.shape[0]
    x, p = native_axes(N)
    px = center[0] + np.linspace(-bound, bound, n)
    pp = center[1] + np.linspace(-bound, bound, n)
    if px[0] < x[0] or px[-1] > x[-1] or pp[0] < p[0] or pp[-1] > p[-1]:
        raise ValueError("grid outside the native grid")
    ix, fx = _weights(x, px)
    ip, fp = _weights(p, pp)
    W = np.asarray(W, dtype=np.float64)
    top = W[ip][:, ix] * (1 - fx) + W[ip][:, ix + 1] * fx
    bot = W[ip + 1][:, ix] * (1 - fx) + W[ip + 1][:, ix + 1] * fx
    return top * (1 - fp)[:, None] + bot * fp[:, None]
