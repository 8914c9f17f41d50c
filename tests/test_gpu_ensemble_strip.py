"""Ensembles on the strip kernels (vp_strip.cu: one launch over all instances' 128-column groups and
runs of bands, then a field launch per step) against the float64 oracle and the ensemble's tile
kernels, with the configuration-4 shapes (nx in {64, 128, 256}, nv in {128, 256, 512}).

Bars (max-norm relative error): float32 1e-5 forward and adjoint, as for the tile kernels.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import vp_oracle as O
from warp_vp_solver_b200 import make_mesh
from warp_vp_solver_b200.ensemble import Ensemble
from warp_vp_solver_b200.workloads import fourier_coefficients, fourier_field, two_stream

pytestmark = pytest.mark.gpu

SHAPES = [(64, 128), (128, 256), (256, 512), (64, 512), (256, 128), (128, 128), (256, 256)]


def _instances(seed, amp=1e-2):
    rng = np.random.default_rng(seed)
    meshes, feqs, fivs, Hs = [], [], [], []
    for i, (nx, nv) in enumerate(SHAPES):
        m = make_mesh(10.0 * np.pi, 6.0, nx, nv)
        f_eq, f_iv = two_stream(m, mu=float(rng.uniform(2.0, 3.0)), eps=float(rng.uniform(1e-4, 1e-2)))
        meshes.append(m)
        feqs.append(f_eq)
        fivs.append(f_iv)
        Hs.append(fourier_field(fourier_coefficients(8, amp, seed + i), m.xs, 2 * np.pi / m.period_x))
    return meshes, feqs, fivs, Hs


def _run(ens, fivs, Hs, T, dt):
    H = ens.pack_rows(Hs)
    out = ens.forward(ens.pack_cells(fivs), H, T, want_tape=True)
    g_ee = torch.full((ens.n * T,), dt, dtype=torch.float32, device=ens.device)
    g_Eh = torch.as_tensor(np.random.default_rng(5).standard_normal(ens.total_rows * T), dtype=torch.float32,
                           device=ens.device)
    g_fiv, g_H = ens.backward(H, T, out["tape"], g_E_hist=g_Eh, g_ee_hist=g_ee)
    torch.cuda.synchronize()
    return out, g_fiv, g_H, g_Eh


@pytest.mark.parametrize("amp", [1e-2, 0.5], ids=["weak", "strong"])
def test_ensemble_strip_matches_oracle_and_tile_kernels(amp, record_error):
    T, dt = 9, 0.05
    meshes, feqs, fivs, Hs = _instances(21, amp)
    ens = Ensemble(meshes, dt, feqs)
    cfg = ens.get_config()
    assert cfg["strip"] == 1 and cfg["strip_ctas"] > 0, cfg
    out, g_fiv, g_H, g_Eh = _run(ens, fivs, Hs, T, dt)
    worst_f = worst_b = 0.0
    for i, m in enumerate(meshes):
        g = O.grid_from(m)
        ref = O.delta_forward(g, dt, feqs[i], fivs[i], Hs[i], T)
        errs = [O.rel_err(ens.cells_of(out["f_final"], i).cpu().numpy(), ref[0]),
                O.rel_err(ens.hist_of(out["E_hist"], i, T).cpu().numpy(), ref[2]),
                O.rel_err(ens.ee_of(out["ee_hist"], i, T).cpu().numpy(), ref[3])]
        worst_f = max(worst_f, *errs)
        gEh_i = ens.hist_of(g_Eh, i, T).cpu().numpy().astype(np.float64)
        rf, rH = O.delta_backward(g, dt, feqs[i], fivs[i], Hs[i], T, np.zeros((m.nx, m.nv)), None, gEh_i,
                                  np.full(T, dt))
        worst_b = max(worst_b, O.rel_err(ens.cells_of(g_fiv, i).cpu().numpy(), rf),
                      O.rel_err(ens.rows_of(g_H, i).cpu().numpy(), rH))
    record_error(f"ensemble strip C4 shapes H{amp} f32 forward", worst_f, 1e-5)
    record_error(f"ensemble strip C4 shapes H{amp} f32 adjoint", worst_b, 1e-5)
    assert worst_f < 1e-5 and worst_b < 1e-5, (worst_f, worst_b)
    # the tile kernels on the same ensemble agree to rounding
    ens.set_config(strip=0)
    assert ens.get_config()["strip"] == 0
    out2, g_fiv2, g_H2, _ = _run(ens, fivs, Hs, T, dt)
    assert O.rel_err(out["ee_hist"].cpu().numpy(), out2["ee_hist"].cpu().numpy()) < 1e-5
    assert O.rel_err(g_H.cpu().numpy(), g_H2.cpu().numpy()) < 1e-5


def test_ensemble_strip_is_deterministic_and_graph_replay_matches_eager():
    T, dt = 6, 0.05
    meshes, feqs, fivs, Hs = _instances(33)
    ens = Ensemble(meshes, dt, feqs)
    assert ens.get_config()["strip"] == 1
    a = _run(ens, fivs, Hs, T, dt)
    b = _run(ens, fivs, Hs, T, dt)
    assert torch.equal(a[0]["f_final"], b[0]["f_final"]) and torch.equal(a[2], b[2])
    f_iv, H = ens.pack_cells(fivs), ens.pack_rows(Hs)
    eager = ens.forward(f_iv, H, T, want_tape=True)
    g_ee = torch.full((ens.n * T,), dt, dtype=torch.float32, device=ens.device)
    g_fiv, g_H = ens.backward(H, T, eager["tape"], g_ee_hist=g_ee)
    graph = ens.capture(T, adjoint=True)
    graph.f_iv.copy_(f_iv)
    graph.H.copy_(H)
    graph.g_ee_hist.copy_(g_ee)
    graph.replay()
    torch.cuda.synchronize()
    assert torch.equal(graph.out["ee_hist"], eager["ee_hist"])
    assert torch.equal(graph.g_f_iv, g_fiv) and torch.equal(graph.g_H, g_H)


def test_ensemble_strip_not_used_where_an_instance_does_not_qualify():
    m1 = make_mesh(10.0 * np.pi, 6.0, 64, 128)
    m2 = make_mesh(10.0 * np.pi, 6.0, 48, 96)   # nv not a multiple of 128
    f1, _ = two_stream(m1, mu=2.4, eps=1e-3)
    f2, _ = two_stream(m2, mu=2.4, eps=1e-3)
    ens = Ensemble([m1, m2], 0.05, [f1, f2])
    assert ens.get_config()["strip"] == 0
    with pytest.raises(ValueError):
        ens.set_config(strip=1)
