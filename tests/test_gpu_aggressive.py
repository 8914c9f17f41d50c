"""The merged-Strang (aggressive) scheme on the GPU against the reference's own aggressive
loops (golden vectors recorded from solver.py:618-736 and 1111-1338).

Bars as for the Strang path (max-norm relative error): float32 1e-5 forward, 1e-4 adjoint;
float64 1e-11 forward, 1e-10 adjoint.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import vp_oracle as O
from conftest import load_golden
from warp_vp_solver_b200 import WarpVlasovPoissonSolver

pytestmark = pytest.mark.gpu

CASES = load_golden("aggressive")
FIELDS = ("f_final", "f_hist", "E_hist", "ee_hist")
TOL_FWD = {torch.float64: 1e-11, torch.float32: 1e-5}
TOL_BWD = {torch.float64: 1e-10, torch.float32: 1e-4}


def _dt_id(d):
    return "f32" if d == torch.float32 else "f64"


@pytest.mark.parametrize("every", [1, 2])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64], ids=_dt_id)
@pytest.mark.parametrize("case", CASES, ids=lambda c: c.name)
def test_aggressive_matches_reference_golden(case, dtype, every):
    s = WarpVlasovPoissonSolver(case.mesh, float(case["dt"]), case["f_eq"], aggressive=True,
                                aggressive_layout=str(case["layout"]), dtype=dtype,
                                checkpoint_every=every)
    assert s.plan.merged
    out = s.run_forward(case["f_iv"], case["H"], float(case["t_final"]))
    for arr, name in zip(out, FIELDS):
        err = O.rel_err(arr, case[name])
        assert err < TOL_FWD[dtype], f"{case.name}:{name} rel err {err:.2e}"
    g_f, g_H = s._run_backward(case["f_iv"], case["H"], float(case["t_final"]), None,
                               case["g_f_final"], case["g_f_hist"], case["g_E_hist"],
                               case["g_ee_hist"])
    e1, e2 = O.rel_err(g_f, case["g_f_iv"]), O.rel_err(g_H, case["g_H"])
    assert e1 < TOL_BWD[dtype] and e2 < TOL_BWD[dtype], f"{case.name}: g_f {e1:.2e} g_H {e2:.2e}"


def test_aggressive_close_to_strang(small_mesh):
    """The merged scheme is a different discretisation (X(dt/2) X(dt/2) != X(dt)) whose f_final,
    E_hist and ee_hist stay within 1e-7 of the Strang path at dt = 0.001 over 5 steps (the
    reference's own bar, tests/test_aggressive.py:257-266), and f_hist[-1] == f_final."""
    m = small_mesh
    f_eq = np.exp(-0.5 * m.V ** 2) / np.sqrt(2.0 * np.pi)
    f0 = f_eq * (1.0 + 0.01 * np.cos(m.X))
    H = np.zeros(m.nx)
    a = WarpVlasovPoissonSolver(m, 0.001, f_eq, aggressive=True, dtype=torch.float64)
    b = WarpVlasovPoissonSolver(m, 0.001, f_eq, dtype=torch.float64)
    fa, fha, Ea, eea = a.run_forward(f0, H, 0.005)
    fb, _, Eb, eeb = b.run_forward(f0, H, 0.005)
    np.testing.assert_allclose(fa, fb, atol=1e-7, rtol=1e-7)
    np.testing.assert_allclose(Ea, Eb, atol=1e-7, rtol=1e-7)
    np.testing.assert_allclose(eea, eeb, atol=1e-7, rtol=1e-7)
    assert not np.array_equal(fha[0], b.run_forward(f0, H, 0.005)[1][0])
    np.testing.assert_array_equal(fha[-1], fa)


def test_aggressive_autograd_matches_oracle():
    c = CASES[0]
    s = WarpVlasovPoissonSolver(c.mesh, float(c["dt"]), c["f_eq"], aggressive=True,
                                dtype=torch.float64)
    f0 = torch.tensor(c["f_iv"], device="cuda", requires_grad=True)
    H = torch.tensor(c["H"], device="cuda", requires_grad=True)
    f_final, f_hist, E_hist, ee = s.run_forward_torch(f0, H, float(c["t_final"]))
    J = (ee * float(c["dt"])).sum() + (E_hist ** 2).sum()
    J.backward()
    T = int(c["n_steps"])
    g = c.grid
    fwd = O.run_forward_aggressive(g, float(c["dt"]), c["f_eq"], c["f_iv"], c["H"], float(c["t_final"]))
    gf, gH = O.run_backward_aggressive(g, float(c["dt"]), c["f_eq"], c["f_iv"], c["H"],
                                       float(c["t_final"]), fwd[1], np.zeros_like(c["f_iv"]),
                                       np.zeros((T, g.nx, g.nv)), 2.0 * fwd[2],
                                       np.full(T, float(c["dt"])))
    assert O.rel_err(f0.grad.cpu().numpy(), gf) < 1e-10
    assert O.rel_err(H.grad.cpu().numpy(), gH) < 1e-10
