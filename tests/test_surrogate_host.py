"""Host-side pieces of the surrogate and of ensemble sharding, on CPU: the Fourier basis and
trapezoid weights against their definitions, the Adam loop against torch.optim.Adam, and the
longest-processing-time shard assignment."""

from __future__ import annotations

import numpy as np
import torch

from warp_vp_solver_b200 import make_mesh
from warp_vp_solver_b200.sharding import lpt_shards, shard_loads
from warp_vp_solver_b200.surrogate import adam_loop, fourier_basis, trapezoid_weights
from warp_vp_solver_b200.utils import external_electric_field
from warp_vp_solver_b200.workloads import make_ensemble_workload


def test_fourier_basis_matches_external_field():
    m = make_mesh(10 * np.pi, 6.0, 64, 32)
    c = np.random.default_rng(0).standard_normal((2, 16))
    B = fourier_basis(m.xs, 0.2, 16)
    H = external_electric_field(torch.tensor(c), m, 0.2).numpy()
    np.testing.assert_allclose(B @ c.reshape(-1), H, rtol=1e-12, atol=1e-12)


def test_trapezoid_weights():
    y = np.random.default_rng(1).standard_normal(37)
    assert abs((trapezoid_weights(37, 0.05) * y).sum() - np.trapezoid(y, dx=0.05)) < 1e-14
    assert trapezoid_weights(1, 0.05)[0] == 0.0


def test_adam_loop_matches_torch_adam():
    A = torch.tensor(np.random.default_rng(2).standard_normal((6, 6)))
    Q = A @ A.T + torch.eye(6)
    fun = lambda c: (0.5 * c.double() @ Q @ c.double(), (Q @ c.double()).float())  # noqa: E731
    c0 = torch.ones(6)
    _, _, hist = adam_loop(fun, c0, 1e-2, 50, lambda h: False)
    t = c0.clone().double().requires_grad_(True)
    opt = torch.optim.Adam([t], lr=1e-2)
    ref = []
    for _ in range(50):
        opt.zero_grad()
        J = 0.5 * t @ Q @ t
        ref.append(float(J.detach()))
        J.backward()
        opt.step()
    np.testing.assert_allclose(hist, ref, rtol=1e-5)


def test_lpt_shards_cover_and_balance():
    wl = make_ensemble_workload("c4", 256, seed=0)
    costs = [m.nx * m.nv for m in wl.meshes]
    for n in (1, 2, 3, 8):
        shards = lpt_shards(costs, n)
        assert sorted(i for s in shards for i in s) == list(range(len(costs)))
        loads = shard_loads(costs, shards)
        # LPT: no rank exceeds the mean by more than the largest single instance
        assert max(loads) - sum(loads) / n <= max(costs)
    assert lpt_shards(costs, 4) == lpt_shards(costs, 4)
