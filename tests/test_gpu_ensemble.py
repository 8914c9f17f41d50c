"""Ensembles of uneven instances (one persistent launch per step) against the reference's golden
vectors, the float64 oracle and the single-instance solver.

Bars (max-norm relative error): float32 1e-5 forward, 1e-5 adjoint (about ten times the largest
adjoint error measured on B200); float64 1e-11 forward, 1e-10 adjoint.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import vp_oracle as O
from conftest import BACKWARD_CASES, FORWARD_CASES, two_stream_state
from warp_vp_solver_b200 import WarpVlasovPoissonSolver, make_mesh
from warp_vp_solver_b200.ensemble import Ensemble, packed_offsets
from warp_vp_solver_b200.workloads import fourier_coefficients, fourier_field

pytestmark = pytest.mark.gpu

TOL_FWD = {torch.float64: 1e-11, torch.float32: 1e-5}
# float32 adjoint: at most 6.3e-7 measured on B200
TOL_BWD = {torch.float64: 1e-10, torch.float32: 1e-5}
DTYPES = [torch.float32, torch.float64]


def _dt_id(d):
    return "f32" if d == torch.float32 else "f64"


def _groups(cases):
    by_t = {}
    for c in cases:
        by_t.setdefault(int(c["n_steps"]), []).append(c)
    return sorted(by_t.items())


FWD_GROUPS = _groups(FORWARD_CASES)
BWD_GROUPS = _groups(BACKWARD_CASES)


def _ensemble(cases, dtype):
    return Ensemble([c.mesh for c in cases], [float(c["dt"]) for c in cases],
                    [c["f_eq"] for c in cases], dtype=dtype)


@pytest.mark.parametrize("dtype", DTYPES, ids=_dt_id)
@pytest.mark.parametrize("group", FWD_GROUPS, ids=lambda g: f"T{g[0]}x{len(g[1])}")
def test_ensemble_forward_matches_reference_golden(group, dtype):
    T, cases = group
    ens = _ensemble(cases, dtype)
    out = ens.forward(ens.pack_cells([c["f_iv"] for c in cases]),
                      ens.pack_rows([c["H"] for c in cases]), T)
    for i, c in enumerate(cases):
        got = {"f_final": ens.cells_of(out["f_final"], i).cpu().numpy(),
               "E_hist": ens.hist_of(out["E_hist"], i, T).cpu().numpy(),
               "ee_hist": ens.ee_of(out["ee_hist"], i, T).cpu().numpy()}
        for name, arr in got.items():
            if c.name.startswith("fwd_equilibrium") and name != "f_final":
                assert np.abs(arr).max() <= 1e-12
                continue
            err = O.rel_err(arr, c[name])
            assert err < TOL_FWD[dtype], f"{c.name}:{name} rel err {err:.2e}"


@pytest.mark.parametrize("dtype", DTYPES, ids=_dt_id)
@pytest.mark.parametrize("group", BWD_GROUPS, ids=lambda g: f"T{g[0]}x{len(g[1])}")
def test_ensemble_backward_matches_oracle(group, dtype, record_error):
    """Adjoint with the golden cotangents on f_final, E and ee (the ensemble API has no f_hist
    cotangent), checked against the float64 delta-f oracle."""
    T, cases = group
    ens = _ensemble(cases, dtype)
    H = ens.pack_rows([c["H"] for c in cases])
    out = ens.forward(ens.pack_cells([c["f_iv"] for c in cases]), H, T, want_tape=True)
    g_fiv, g_H = ens.backward(H, T, out["tape"],
                              g_f_final=ens.pack_cells([c["g_f_final"] for c in cases], ens.dtype),
                              g_E_hist=ens.pack_hist([c["g_E_hist"] for c in cases], T),
                              g_ee_hist=torch.cat([torch.as_tensor(c["g_ee_hist"]) for c in cases]))
    for i, c in enumerate(cases):
        ref_f, ref_H = O.delta_backward(c.grid, float(c["dt"]), c["f_eq"], c["f_iv"], c["H"], T,
                                        c["g_f_final"], None, c["g_E_hist"], c["g_ee_hist"])
        e1 = O.rel_err(ens.cells_of(g_fiv, i).cpu().numpy(), ref_f)
        e2 = O.rel_err(ens.rows_of(g_H, i).cpu().numpy(), ref_H)
        if dtype == torch.float32:
            record_error(f"ensemble {c.name} f32 adjoint", max(e1, e2), TOL_BWD[dtype])
        assert e1 < TOL_BWD[dtype] and e2 < TOL_BWD[dtype], f"{c.name}: g_f {e1:.2e} g_H {e2:.2e}"


def _uneven(n, seed, nxs=(16, 32, 64), nvs=(32, 64, 128)):
    rng = np.random.default_rng(seed)
    meshes, feqs, fivs, Hs = [], [], [], []
    for i in range(n):
        m = make_mesh(10.0 * np.pi, 6.0, int(rng.choice(nxs)), int(rng.choice(nvs)))
        f_eq, f_iv = two_stream_state(m, mu=float(rng.uniform(2.0, 3.0)),
                                      eps=float(rng.uniform(1e-4, 1e-2)))
        H = fourier_field(fourier_coefficients(8, 1e-2, seed * 1000 + i), m.xs, 2 * np.pi / m.period_x)
        meshes.append(m), feqs.append(f_eq), fivs.append(f_iv), Hs.append(H)
    return meshes, feqs, fivs, Hs


@pytest.mark.parametrize("dtype", DTYPES, ids=_dt_id)
def test_uneven_ensemble_matches_oracle_and_single_solver(dtype):
    T, dt = 12, 0.05
    meshes, feqs, fivs, Hs = _uneven(11, seed=3)
    ens = Ensemble(meshes, dt, feqs, dtype=dtype)
    H = ens.pack_rows(Hs)
    out = ens.forward(ens.pack_cells(fivs), H, T, want_tape=True)
    g_ee = torch.full((ens.n * T,), dt, dtype=dtype, device=ens.device)
    g_fiv, g_H = ens.backward(H, T, out["tape"], g_ee_hist=g_ee)
    for i, m in enumerate(meshes):
        g = O.grid_from(m)
        ref = O.delta_forward(g, dt, feqs[i], fivs[i], Hs[i], T)
        assert O.rel_err(ens.cells_of(out["f_final"], i).cpu().numpy(), ref[0]) < TOL_FWD[dtype]
        assert O.rel_err(ens.hist_of(out["E_hist"], i, T).cpu().numpy(), ref[2]) < TOL_FWD[dtype]
        assert O.rel_err(ens.ee_of(out["ee_hist"], i, T).cpu().numpy(), ref[3]) < TOL_FWD[dtype]
        rf, rH = O.delta_backward(g, dt, feqs[i], fivs[i], Hs[i], T, np.zeros((m.nx, m.nv)),
                                  None, np.zeros((T, m.nx)), np.full(T, dt))
        assert O.rel_err(ens.cells_of(g_fiv, i).cpu().numpy(), rf) < TOL_BWD[dtype]
        assert O.rel_err(ens.rows_of(g_H, i).cpu().numpy(), rH) < TOL_BWD[dtype]
        # the single-instance solver on the same instance
        s = WarpVlasovPoissonSolver(m, dt, feqs[i], dtype=dtype)
        single = s.run_forward(fivs[i], Hs[i], T * dt)
        assert O.rel_err(ens.ee_of(out["ee_hist"], i, T).cpu().numpy(), single[3]) < TOL_FWD[dtype]


def test_ensemble_offsets_and_step_count():
    meshes, feqs, _, _ = _uneven(5, seed=1)
    ens = Ensemble(meshes, 0.05, feqs)
    co, ro, tc, tr = packed_offsets(ens.shapes)
    np.testing.assert_array_equal(ens.cell_offsets, co)
    np.testing.assert_array_equal(ens.row_offsets, ro)
    assert (ens.total_cells, ens.total_rows) == (tc, tr)
    assert ens.num_steps(5.0) == 100
    mixed = Ensemble(meshes[:2], [0.05, 0.03], feqs[:2])
    with pytest.raises(ValueError):
        mixed.num_steps(5.0)


def test_ensemble_autograd_matches_single_instance_autograd():
    T, dt = 8, 0.05
    meshes, feqs, fivs, Hs = _uneven(4, seed=7)
    ens = Ensemble(meshes, dt, feqs)
    f_iv = ens.pack_cells(fivs).requires_grad_(True)
    H = ens.pack_rows(Hs).requires_grad_(True)
    _, E_hist, ee = ens.run_forward_torch(f_iv, H, T)
    J = (ee.double() * dt).sum() + 0.1 * (E_hist.double() ** 2).sum()
    J.backward()
    for i, m in enumerate(meshes):
        s = WarpVlasovPoissonSolver(m, dt, feqs[i])
        fi = torch.as_tensor(fivs[i], device="cuda").requires_grad_(True)
        Hi = torch.as_tensor(Hs[i], device="cuda", dtype=torch.float32).requires_grad_(True)
        _, _, Ei, eei = s.run_forward_torch(fi, Hi, T * dt)
        Ji = (eei.double() * dt).sum() + 0.1 * (Ei.double() ** 2).sum()
        Ji.backward()
        assert O.rel_err(ens.cells_of(f_iv.grad, i).cpu().numpy(), fi.grad.cpu().numpy()) < 1e-4
        assert O.rel_err(ens.rows_of(H.grad, i).cpu().numpy(), Hi.grad.cpu().numpy()) < 1e-4


def test_ensemble_graph_replay_matches_eager():
    T, dt = 10, 0.05
    meshes, feqs, fivs, Hs = _uneven(6, seed=11)
    ens = Ensemble(meshes, dt, feqs)
    f_iv, H = ens.pack_cells(fivs), ens.pack_rows(Hs)
    eager = ens.forward(f_iv, H, T, want_tape=True)
    g_ee = torch.full((ens.n * T,), dt, dtype=torch.float32, device=ens.device)
    g_fiv, g_H = ens.backward(H, T, eager["tape"], g_ee_hist=g_ee)
    graph = ens.capture(T, adjoint=True)
    graph.f_iv.copy_(f_iv)
    graph.H.copy_(H)
    graph.g_ee_hist.copy_(g_ee)
    for _ in range(2):
        graph.replay()
        torch.cuda.synchronize()
        assert torch.equal(graph.out["ee_hist"], eager["ee_hist"])
        assert torch.equal(graph.out["f_final"], eager["f_final"])
        assert torch.equal(graph.g_f_iv, g_fiv)
        assert torch.equal(graph.g_H, g_H)


def test_ensemble_rejects_bad_arguments():
    meshes, feqs, fivs, Hs = _uneven(2, seed=2)
    ens = Ensemble(meshes, 0.05, feqs)
    with pytest.raises(ValueError):
        ens.forward(ens.pack_cells(fivs), ens.pack_rows(Hs), 0)
    with pytest.raises(ValueError):
        ens.forward(ens.pack_cells(fivs)[:-1], ens.pack_rows(Hs), 3)
    with pytest.raises(ValueError):
        Ensemble(meshes, 0.05, feqs[:1])


def test_sharded_ensemble_entry_point_solves_on_the_device():
    """solve_sharded_ensemble with its default per-shard solve (one Ensemble on this GPU, a
    single rank here) against the float64 oracle per instance: energy and field histories and
    dJ/dH of J = trapezoid(ee, dt)."""
    from warp_vp_solver_b200.sharding import solve_sharded_ensemble
    T, dt = 10, 0.05
    meshes, feqs, fivs, Hs = _uneven(6, seed=21)
    res = solve_sharded_ensemble(meshes, dt, feqs, fivs, Hs, T, want_grad=True)
    for i, m in enumerate(meshes):
        g = O.grid_from(m)
        ref = O.delta_forward(g, dt, feqs[i], fivs[i], Hs[i], T)
        _, rH = O.delta_backward(g, dt, feqs[i], fivs[i], Hs[i], T, np.zeros((m.nx, m.nv)), None,
                                 np.zeros((T, m.nx)), O.trapezoid_time_weights(T, dt))
        assert O.rel_err(res[i]["ee_hist"], ref[3]) < 1e-5
        assert O.rel_err(res[i]["E_hist"], ref[2]) < 1e-5
        assert O.rel_err(res[i]["g_H"], rH) < 1e-4
