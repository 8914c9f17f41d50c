"""Properties the reference's own tests assert, checked on the oracle (CPU).

Sources: tests/test_poisson.py, tests/test_kernels.py, tests/test_solver.py of the reference.
These guard the oracle itself; the GPU tests then compare the CUDA path against it.
"""

from __future__ import annotations

import numpy as np

import vp_oracle as O
from conftest import two_stream_state


def _grid64():
    return O.make_grid(10.0 * np.pi, 6.0, 64, 64)


def _state(g, **kw):
    V, X = np.meshgrid(g.vs, g.xs)

    class M:
        pass

    m = M()
    m.V, m.X = V, X
    return two_stream_state(m, **kw)


def test_poisson_zero_and_dc():
    assert np.abs(O.solve_poisson(np.zeros(64), 2 * np.pi)).max() < 1e-15
    rho = np.random.default_rng(0).standard_normal(64)
    E = O.solve_poisson(rho, 2 * np.pi)
    assert abs(np.fft.fft(E)[0]) < 1e-12


def test_poisson_single_mode():
    xs = np.linspace(0.0, 2 * np.pi, 64, endpoint=False)
    E = O.solve_poisson(np.sin(2.0 * xs), 2 * np.pi)
    np.testing.assert_allclose(E, np.cos(2.0 * xs) / 2.0, atol=1e-12)


def test_poisson_adjoint_inner_product():
    rng = np.random.default_rng(0)
    rho, gE = rng.standard_normal(64), rng.standard_normal(64)
    lhs = np.dot(O.solve_poisson(rho, 2 * np.pi), gE)
    rhs = np.dot(rho, O.solve_poisson_adjoint(gE, 2 * np.pi))
    np.testing.assert_allclose(lhs, rhs, rtol=1e-12, atol=1e-12)


def test_x_and_v_adjoint_inner_products():
    g = _grid64()
    _, f = _state(g)
    rng = np.random.default_rng(3)
    go = rng.standard_normal(f.shape)
    lhs = np.sum(O.semilag_x(f, g, 0.07) * go)
    rhs = np.sum(f * O.semilag_x_adjoint(go, g, 0.07))
    np.testing.assert_allclose(lhs, rhs, rtol=1e-12)
    E = 0.01 * rng.standard_normal(g.nx)
    gi, _ = O.semilag_v_adjoint(go, f, E, g, 0.05)
    np.testing.assert_allclose(np.sum(O.semilag_v(f, E, g, 0.05) * go), np.sum(f * gi), rtol=1e-12)


def test_v_adjoint_field_gradient_fd():
    g = _grid64()
    _, f = _state(g)
    rng = np.random.default_rng(5)
    go = rng.standard_normal(f.shape)
    E = 0.01 * rng.standard_normal(g.nx)
    _, gE = O.semilag_v_adjoint(go, f, E, g, 0.05)
    eps, k = 1e-6, 3
    Ep, Em = E.copy(), E.copy()
    Ep[k] += eps
    Em[k] -= eps
    fd = np.sum((O.semilag_v(f, Ep, g, 0.05) - O.semilag_v(f, Em, g, 0.05)) / (2 * eps) * go)
    np.testing.assert_allclose(gE[k], fd, rtol=1e-5, atol=1e-7)


def test_mass_conservation_and_equilibrium():
    g = O.make_grid(2 * np.pi, 6.0, 16, 32)
    V, X = np.meshgrid(g.vs, g.xs)
    f_eq = np.exp(-0.5 * V ** 2)
    f0 = f_eq * (1 + 1e-3 * np.cos(X))
    ff, _, _, _ = O.run_forward(g, 0.001, f_eq, f0, np.zeros(16), 10 * 0.001)

    def mass(f):
        return np.trapezoid(np.trapezoid(f, g.xs, axis=0), g.vs, axis=0)

    np.testing.assert_allclose(mass(ff), mass(f0), rtol=1e-5, atol=1e-7)
    fd, _, Ed, eed = O.delta_forward(g, 0.05, f_eq, f_eq.copy(), np.zeros(16), 5)
    assert np.array_equal(fd, f_eq)
    assert np.abs(Ed).max() == 0.0 and np.abs(eed).max() == 0.0


def test_backward_matches_central_differences():
    """dJ/dH of J = trapezoid(ee, dt) against central differences (test_solver.py:155-176)."""
    g = O.make_grid(10.0 * np.pi, 6.0, 32, 32)
    V, X = np.meshgrid(g.vs, g.xs)
    f_eq = (np.exp(-0.5 * (V - 2.4) ** 2) + np.exp(-0.5 * (V + 2.4) ** 2)) / (2 * np.sqrt(2 * np.pi))
    f0 = (1 + 1e-3 * np.cos(0.2 * X)) * f_eq
    rng = np.random.default_rng(42)
    H = 0.01 * rng.standard_normal(g.nx)
    dt, T = 0.05, 8
    w = O.trapezoid_time_weights(T, dt)

    def J(Hv):
        return float(np.dot(O.delta_forward(g, dt, f_eq, f0, Hv, T)[3], w))

    _, gH = O.delta_backward(g, dt, f_eq, f0, H, T, np.zeros_like(f0), None, None, w)
    d = rng.standard_normal(g.nx)
    eps = 1e-6
    fd = (J(H + eps * d) - J(H - eps * d)) / (2 * eps)
    np.testing.assert_allclose(np.dot(gH, d), fd, rtol=1e-6)
