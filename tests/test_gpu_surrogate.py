"""The learned surrogate end to end on a small two-stream set-up: data from the ensemble solver,
training by the tensor-core MLP kernels, and what the trained network gains: from the same
random initial control, the warm-started loop reaches the plain adjoint loop's J* (within 1%)
with a fraction of the true forward+adjoint evaluations."""

from __future__ import annotations

import pytest

from warp_vp_solver_b200.surrogate import c5_setup, run_comparison

pytestmark = pytest.mark.gpu


def test_surrogate_warm_start_needs_fewer_adjoint_evaluations():
    setup = c5_setup(nx=64, nv=64, n_steps=50, n_modes=8, eps=1e-2)
    res = run_comparison(setup, n_samples=1024, coeff_std=0.05, train_steps=1000, seeds=[11, 12],
                         batch=256, sur_iters=150, lr_sur=3e-3)
    assert res["mlp_status"] == 0
    # the network learned the map: held-out error well below predicting the mean history
    assert res["holdout_mae_log_ee"] < 0.5 * res["holdout_mae_mean_predictor"]
    for r in res["runs"]:
        assert r["warm_reached"], r
        assert r["plain_evals_to_target"] is not None
        assert 3 * r["warm_evals"] <= r["plain_evals_to_target"], r
