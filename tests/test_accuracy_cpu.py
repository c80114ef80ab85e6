"""CPU checks of the accuracy helpers used by the mixed-form measurements."""

import math

import numpy as np
import torch

from cvdv_b200.accuracy import compare_states, native_axes, wigner_grid


def test_wigner_grid_exact_on_bilinear_functions():
    N = 256
    x, p = native_axes(N)
    P, X = np.meshgrid(p, x, indexing="ij")
    W = 0.3 + 0.5 * X - 0.2 * P + 0.07 * X * P
    g = wigner_grid(W, n=64, bound=6.0)
    pts = np.linspace(-6, 6, 64)
    Pg, Xg = np.meshgrid(pts, pts, indexing="ij")
    np.testing.assert_allclose(g, 0.3 + 0.5 * Xg - 0.2 * Pg + 0.07 * Xg * Pg, atol=1e-12)


def test_wigner_grid_bound_outside_native_grid():
    import pytest
    with pytest.raises(ValueError):
        wigner_grid(np.zeros((16, 16)), n=8, bound=6.0)  # native x spans only +-3.9


def test_compare_states_known_values():
    rng = np.random.default_rng(0)
    a = rng.standard_normal(1000) + 1j * rng.standard_normal(1000)
    b = a * np.exp(0.3j)  # global phase: fidelity 1
    r = compare_states(torch.from_numpy(a), torch.from_numpy(b.astype(np.complex64)), chunk=128)
    assert r["infidelity"] < 1e-12
    c = a.copy()
    c[0] += 1.0
    r = compare_states(torch.from_numpy(a), torch.from_numpy(c), chunk=300)
    assert abs(r["max_abs_err"] - 1.0) < 1e-12
    assert abs(r["rel_l2"] - 1.0 / np.linalg.norm(a)) < 1e-12
    ov = abs(np.vdot(a, c)) ** 2 / (np.vdot(a, a).real * np.vdot(c, c).real)
    assert math.isclose(r["infidelity"], 1 - ov, rel_tol=1e-9)
