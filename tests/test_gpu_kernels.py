"""Single-stage operators on the device against the reference's kernels (golden vectors) and
the reference's kernel-level properties (tests/test_kernels.py, tests/test_poisson.py)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import vp_oracle as O
from warp_vp_solver_b200 import WarpVlasovPoissonSolver, make_mesh
from warp_vp_solver_b200.poisson import solve_poisson, solve_poisson_adjoint

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def kplan(golden_kernels):
    k = golden_kernels
    m = make_mesh(float(k["mesh_length_x"]), float(k["mesh_length_v"]), int(k["mesh_nx"]),
                  int(k["mesh_nv"]))
    s = WarpVlasovPoissonSolver(m, 0.05, k["f_eq"], dtype=torch.float64)
    return s.plan, k


def _np(t):
    return t.double().cpu().numpy()


def test_semilag_x_and_adjoint(kplan):
    p, k = kplan
    assert O.rel_err(_np(p.semilag_x(k["f_iv"], float(k["x_dt"]))), k["x_out"]) < 1e-13
    assert O.rel_err(_np(p.semilag_x(k["xadj_g_out"], float(k["xadj_dt"]), adjoint=True)),
                     k["xadj_g_in"]) < 1e-13
    np.testing.assert_array_equal(_np(p.semilag_x(k["f_iv"], 0.0)), k["f_iv"])


def test_semilag_v_and_adjoint(kplan):
    p, k = kplan
    assert O.rel_err(_np(p.semilag_v(k["f_iv"], k["v_E"], float(k["v_dt"]))), k["v_out"]) < 1e-13
    g_in, g_E = p.semilag_v(k["vadj_g_out"], k["vadj_E"], float(k["vadj_dt"]), adjoint=True,
                            f_in=k["f_iv"])
    assert O.rel_err(_np(g_in), k["vadj_g_in"]) < 1e-13
    assert O.rel_err(_np(g_E), k["vadj_g_E"]) < 1e-11
    np.testing.assert_array_equal(_np(p.semilag_v(k["f_iv"], np.zeros(p.nx), 0.05)), k["f_iv"])


def test_rho_ee_poisson(kplan):
    p, k = kplan
    assert O.rel_err(_np(p.compute_rho(k["f_iv"])), k["rho"]) < 1e-12
    assert abs(_np(p.electric_energy(k["ee_E"]))[0] - k["ee"][0]) < 1e-13 * abs(k["ee"][0])
    assert O.rel_err(_np(p.poisson(k["poisson_rho"])), k["poisson_E"]) < 1e-13
    assert O.rel_err(_np(p.poisson(k["poisson_g_E"], adjoint=True)), k["poisson_adj"]) < 1e-13


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-12), (torch.float32, 2e-6)])
def test_adjoint_dot_products(dtype, tol):
    m = make_mesh(10.0 * np.pi, 6.0, 64, 64)
    rng = np.random.default_rng(3)
    f = rng.standard_normal((64, 64))
    go = rng.standard_normal((64, 64))
    E = 0.01 * rng.standard_normal(64)
    p = WarpVlasovPoissonSolver(m, 0.05, np.ones((64, 64)), dtype=dtype).plan
    lhs = np.sum(_np(p.semilag_x(f, 0.07)) * go)
    rhs = np.sum(f * _np(p.semilag_x(go, 0.07, adjoint=True)))
    assert abs(lhs - rhs) <= tol * np.sum(np.abs(f * go))
    lhs = np.sum(_np(p.semilag_v(f, E, 0.05)) * go)
    rhs = np.sum(f * _np(p.semilag_v(go, E, 0.05, adjoint=True)[0]))
    assert abs(lhs - rhs) <= tol * np.sum(np.abs(f * go))
    rho, gE = rng.standard_normal(64), rng.standard_normal(64)
    lhs = np.dot(_np(p.poisson(rho)), gE)
    rhs = np.dot(rho, _np(p.poisson(gE, adjoint=True)))
    assert abs(lhs - rhs) <= 10 * tol * np.sum(np.abs(rho)) * np.sum(np.abs(gE))


@pytest.mark.parametrize("nx", [64, 256, 24])
def test_poisson_analytic_mode(nx):
    period = 2.0 * np.pi
    xs = np.linspace(0.0, period, nx, endpoint=False)
    E = solve_poisson(np.sin(2.0 * xs), period, dtype=torch.float64)
    np.testing.assert_allclose(E, np.cos(2.0 * xs) / 2.0, atol=1e-12)
    assert np.abs(solve_poisson(np.zeros(nx), period)).max() == 0.0
    rng = np.random.default_rng(0)
    g = rng.standard_normal(nx)
    assert O.rel_err(solve_poisson_adjoint(g, period, dtype=torch.float64),
                     O.solve_poisson_adjoint(g, period)) < 1e-12
