"""The learned surrogate end to end: data from the ensemble solver, training by the tensor-core MLP
kernels, and what the trained network gains. From the same random initial control, the
warm-started loop (surrogate search, then true-gradient Adam) reaches the plain adjoint loop's J*
(Adam at the reference notebook's step size 1e-3 until J stops improving) within 1% with a
fraction of the true forward+adjoint evaluations and of the wall time. The main case runs at
configuration 5's grid and field (256x256, 100 steps, 16 modes, coefficients of standard
deviation 0.05), with fewer training samples and steps than the benchmark's 4096 x 2000."""

from __future__ import annotations

import pytest

from warp_vp_solver_b200.surrogate import c5_setup, run_comparison

pytestmark = pytest.mark.gpu


def test_surrogate_warm_start_gain_at_the_configuration_grid():
    setup = c5_setup()   # 256x256, dt 0.05, 100 steps, 16 modes
    res = run_comparison(setup, n_samples=2048, coeff_std=0.05, train_steps=1000, seeds=[11, 12, 13],
                         batch=512, sur_iters=150, lr_sur=3e-3, lr_refine=3e-3)
    assert res["mlp_status"] == 0
    # the network learned the map: held-out error well below predicting the mean history
    assert res["holdout_mae_log_ee"] < 0.5 * res["holdout_mae_mean_predictor"]
    for r in res["runs"]:
        assert r["warm_reached"], r
        assert r["plain_evals_to_target"] is not None
        assert 3 * r["warm_evals"] <= r["plain_evals"], r
        assert 3 * r["warm_seconds"] <= r["plain_seconds"], r


def test_surrogate_warm_start_needs_fewer_adjoint_evaluations_small_grid():
    setup = c5_setup(nx=64, nv=64, n_steps=50, n_modes=8, eps=1e-2)
    res = run_comparison(setup, n_samples=1024, coeff_std=0.05, train_steps=1000, seeds=[11, 12],
                         batch=256, sur_iters=150, lr_sur=3e-3)
    assert res["mlp_status"] == 0
    assert res["holdout_mae_log_ee"] < 0.5 * res["holdout_mae_mean_predictor"]
    for r in res["runs"]:
        assert r["warm_reached"], r
        assert r["plain_evals_to_target"] is not None
        assert 3 * r["warm_evals"] <= r["plain_evals_to_target"], r


def test_search_kernel_matches_eager_surrogate_descent():
    """vp_mlp_search (one launch) against Adam driven from the host through the tensor-core MLP's
    forward and input gradient: same starting point, same lr, the best J within 2%, and the
    kernel's reported J equals the surrogate evaluated at its best point."""
    import torch

    from warp_vp_solver_b200.surrogate import (ControlProblem, Surrogate, SurrogateSearch, adam_loop,
                                               generate_dataset)
    setup = c5_setup(nx=64, nv=64, n_steps=30, n_modes=4, eps=1e-2)
    X, Y, _ = generate_dataset(setup, 512, 0.05, seed=0)
    sur = Surrogate(setup.n_inputs, setup.n_steps, max_batch=512, seed=2)
    sur.fit(X, Y, steps=300, batch=256)
    w = ControlProblem(setup).w.float()
    c0 = torch.tensor([0.05, -0.03, 0.02, 0.04, -0.01, 0.03, 0.0, -0.02], device="cuda")
    search = SurrogateSearch(sur, w, lr=3e-3)
    c_k = search.run(c0, 60)
    J_k = float(search.best_J)
    J_at, _ = sur.cost_and_grad(c_k, w)
    assert abs(float(J_at) - J_k) <= 1e-3 * abs(J_k)
    c_e, J_e, _ = adam_loop(lambda c: sur.cost_and_grad(c, w), c0, 3e-3, 60, lambda h: False)
    assert abs(J_k - J_e) <= 0.02 * abs(J_e)
    assert J_k < float(sur.cost_and_grad(c0, w)[0])
