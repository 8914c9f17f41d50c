"""Autotuner on the device: the chosen shape is applied, cached, and gives the oracle's result."""

from __future__ import annotations

import numpy as np
import pytest

import vp_oracle as O
from conftest import two_stream_state
from warp_vp_solver_b200 import WarpVlasovPoissonSolver, make_mesh
from warp_vp_solver_b200.autotune import TuneCache, tune_ensemble
from warp_vp_solver_b200.ensemble import Ensemble

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nx,nv", [(64, 256), (256, 256)])
def test_tune_plan_applies_caches_and_keeps_parity(tmp_path, nx, nv):
    m = make_mesh(10.0 * np.pi, 6.0, nx, nv)
    f_eq, f_iv = two_stream_state(m, eps=1e-2)
    H = 0.05 * np.random.default_rng(0).standard_normal(nx)
    path = str(tmp_path / "tune.json")
    s = WarpVlasovPoissonSolver(m, 0.05, f_eq)
    r = s.autotune(steps=4, cache_path=path)
    assert r["config"] is not None and not r["cached"] and len(r["tried"]) >= 3
    cfg = s.plan.get_config()
    for k, v in r["config"].items():
        assert cfg[k] == v
    out = s.run_forward(f_iv, H, 0.4)
    ref = O.delta_forward(O.grid_from(m), 0.05, f_eq, f_iv, H, 8)
    assert O.rel_err(out[0], ref[0]) < 1e-5 and O.rel_err(out[3], ref[3]) < 1e-5
    s2 = WarpVlasovPoissonSolver(m, 0.05, f_eq)
    r2 = s2.autotune(steps=4, cache_path=path)
    assert r2["cached"] and r2["config"] == r["config"]


def test_tune_ensemble_keeps_parity(tmp_path):
    rng = np.random.default_rng(4)
    meshes, feqs, fivs, Hs = [], [], [], []
    for _ in range(5):
        m = make_mesh(10.0 * np.pi, 6.0, int(rng.choice([16, 32])), int(rng.choice([64, 128])))
        f_eq, f_iv = two_stream_state(m, eps=1e-2)
        meshes.append(m), feqs.append(f_eq), fivs.append(f_iv)
        Hs.append(0.02 * rng.standard_normal(m.nx))
    ens = Ensemble(meshes, 0.05, feqs)
    r = tune_ensemble(ens, steps=3, repeats=1, cache=TuneCache(str(tmp_path / "t.json")), max_candidates=8)
    assert r["config"] is not None
    T = 6
    out = ens.forward(ens.pack_cells(fivs), ens.pack_rows(Hs), T)
    for i, m in enumerate(meshes):
        ref = O.delta_forward(O.grid_from(m), 0.05, feqs[i], fivs[i], Hs[i], T)
        assert O.rel_err(ens.ee_of(out["ee_hist"], i, T).cpu().numpy(), ref[3]) < 1e-5
