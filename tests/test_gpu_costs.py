"""Cost layer on the device: the fused KL(f || f_eq) cost and gradient (vp_kl_divergence) against
the reference's expression (utils.py:53-76) evaluated in torch float64, and through
make_cost_function_kl's gradient."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import vp_oracle as O
from conftest import two_stream_state
from warp_vp_solver_b200 import WarpVlasovPoissonSolver, make_mesh
from warp_vp_solver_b200 import utils as U

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nx,nv", [(32, 64), (64, 128), (24, 40)])
def test_kl_value_and_gradient_match_torch_expression(nx, nv):
    m = make_mesh(10.0 * np.pi, 6.0, nx, nv)
    f_eq, f_iv = two_stream_state(m, eps=0.05)
    s = WarpVlasovPoissonSolver(m, 0.1, f_eq)
    f = torch.tensor(f_iv * (1.0 + 0.1 * np.random.default_rng(nx).random((nx, nv))), device="cuda")
    fd = f.clone().requires_grad_(True)
    v = U.kl_divergence(fd, s)
    v.backward()
    fc = f.cpu().clone().requires_grad_(True)
    ref = U.kl_divergence(fc, s)          # torch expression (CPU tensor)
    ref.backward()
    assert abs(float(v.detach()) - float(ref.detach())) <= 1e-12 * max(1.0, abs(float(ref.detach())))
    assert O.rel_err(fd.grad.cpu().numpy(), fc.grad.numpy()) < 1e-10


def test_kl_cost_gradient_through_the_solver():
    m = make_mesh(10.0 * np.pi, 6.0, 32, 64)
    f_eq, f_iv = two_stream_state(m, eps=1e-2)
    s = WarpVlasovPoissonSolver(m, 0.1, f_eq, dtype=torch.float64)
    k0 = 2 * np.pi / m.period_x
    cost = U.make_cost_function_kl(s, s.run_forward_torch, torch.tensor(f_iv, device="cuda"), k0, 0.5)
    a = torch.tensor(1e-2 * np.random.default_rng(1).standard_normal((2, 3)), device="cuda",
                     requires_grad=True)
    J = cost(a)
    J.backward()
    # the same cost with the torch expression of KL on the device result
    a2 = a.detach().clone().requires_grad_(True)
    H = U.external_electric_field(a2, m, k0)
    f_final = s.run_forward_torch(torch.tensor(f_iv, device="cuda"), H, 0.5)[0]
    J2 = U.kl_divergence(f_final.cpu(), s)
    J2.backward()
    assert abs(float(J.detach()) - float(J2.detach())) <= 1e-12 * max(1.0, abs(float(J2.detach())))
    assert O.rel_err(a.grad.cpu().numpy(), a2.grad.cpu().numpy()) < 1e-9
