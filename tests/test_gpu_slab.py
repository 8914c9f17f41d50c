"""x-slab decomposition on the GPU: the ``vp_slab_*`` calls through ``slab.SlabSolver``.

Every slab of the grid runs on this one device (``LocalRing``: the ranks' launches follow one
another on one stream and the ghost exchanges are device copies; nothing waits on another rank).
A slab's owned rows read exactly the rows the one-grid step reads, with the same per-column
arithmetic and the same column-chunk partial sums, so the slab loops must equal the one-grid
per-column path bit for bit: forward (f_final, f_hist, E_hist, ee_hist) and adjoint (g_f_iv, g_H,
with the checkpointed replay on both sides). Both are also checked against the float64 oracle at
the parity bars (float32 1e-5 forward and 5e-6 adjoint over these short loops; float64 1e-11).
One case runs ``DistRing`` on a one-rank NCCL group."""

from __future__ import annotations

import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist

import vp_oracle as O
from warp_vp_solver_b200 import make_mesh
from warp_vp_solver_b200.plan import Plan
from warp_vp_solver_b200.slab import DistRing, LocalRing, SlabSolver

pytestmark = pytest.mark.gpu

# (length_x, nx, nv, dt, T, dtype, slab counts); the second case shifts columns by up to 2 cells
CASES = [(10 * np.pi, 256, 256, 0.05, 20, torch.float32, (1, 2, 4)),
         (2 * np.pi, 128, 128, 0.1, 12, torch.float32, (2, 3)),
         (2 * np.pi, 128, 128, 0.1, 12, torch.float64, (3,))]
BARS = {torch.float32: (1e-5, 5e-6), torch.float64: (1e-11, 1e-11)}


def _problem(length_x, nx, nv, dt, T, seed=1):
    m = make_mesh(length_x, 6.0, nx, nv)
    f_eq = (np.exp(-0.5 * (m.vs - 2.4) ** 2) + np.exp(-0.5 * (m.vs + 2.4) ** 2)) / (2 * np.sqrt(2 * np.pi))
    rng = np.random.default_rng(seed)
    f_iv = (1.0 + 1e-2 * np.cos(2 * np.pi / length_x * m.X) + 1e-3 * rng.standard_normal((nx, nv))) * f_eq[None, :]
    H = 0.05 * rng.standard_normal(nx)
    gEh = 1e-2 * rng.standard_normal((T, nx))
    gff = 1e-1 * rng.standard_normal((nx, nv))
    return m, f_eq, f_iv, H, gEh, gff


def _one_grid(m, f_eq, f_iv, H, gEh, gee, gff, dt, T, dtype, K):
    plan = Plan(m, dt, np.broadcast_to(f_eq, (m.nx, m.nv)), dtype=dtype)
    plan.set_config(cluster_size=0, stage_rows=0, persist_rows=0, strip_rows=0)
    cfg = plan.get_config()
    assert cfg["cluster_size"] == 0 and cfg["stage_rows"] == 0 and cfg["persist_rows"] == 0
    assert cfg["strip_rows"] == 0
    out = plan.forward(f_iv, H, T, record_history=True, want_tape=True, checkpoint_every=K)
    g_fiv, g_H = plan.backward(H, T, out["tape"], out["every"], g_f_final=gff, g_E_hist=gEh, g_ee_hist=gee)
    torch.cuda.synchronize()
    return {k: out[k].cpu().numpy() for k in ("f_final", "f_hist", "E_hist", "ee_hist")}, \
        g_fiv.cpu().numpy(), g_H.cpu().numpy()


def _slabs(m, f_eq, f_iv, H, gEh, gee, gff, dt, T, dtype, ring, K):
    s = SlabSolver(m, dt, f_eq, ring, dtype=dtype)
    b = s.bounds
    rows = lambda a: {k: a[b[k][0]:b[k][0] + b[k][1]] for k in ring.local}   # noqa: E731
    ff, fh, Eh, eeh = s.run_forward(rows(f_iv), H, T * dt, record_history=True)
    out = s.vjp(rows(f_iv), H, T * dt, g_E_hist=gEh, g_ee_hist=gee, g_f_final_rows=rows(gff), checkpoint_every=K)
    torch.cuda.synchronize()
    join = lambda d, ax=0: np.concatenate([d[k].cpu().numpy() for k in sorted(d)], axis=ax)   # noqa: E731
    return ({"f_final": join(ff), "f_hist": join(fh, 1), "E_hist": Eh.cpu().numpy(), "ee_hist": eeh.cpu().numpy()},
            join(out["g_f_iv"]), out["g_H"].cpu().numpy(), out["ee_hist"].cpu().numpy())


def _check_case(case, rings, record_error):
    length_x, nx, nv, dt, T, dtype, _ = case
    m, f_eq, f_iv, H, gEh, gff = _problem(length_x, nx, nv, dt, T)
    gee = O.trapezoid_time_weights(T, dt)
    K = int(np.ceil(np.sqrt(T)))
    ref_f, ref_gfiv, ref_gH = _one_grid(m, f_eq, f_iv, H, gEh, gee, gff, dt, T, dtype, K)
    g = O.grid_from(m)
    feq2 = np.broadcast_to(f_eq, (nx, nv))
    orc = O.delta_forward(g, dt, feq2, f_iv, H, T)
    o_gfiv, o_gH = O.delta_backward(g, dt, feq2, f_iv, H, T, gff, None, gEh, gee)
    bar_f, bar_g = BARS[dtype]
    tag = f"slab {nx}x{nv} {str(dtype)[6:]}"
    diffs = {}
    for label, ring in rings:
        f, gfiv, gH, ee_vjp = _slabs(m, f_eq, f_iv, H, gEh, gee, gff, dt, T, dtype, ring, K)
        for name, o in (("f_final", orc[0]), ("f_hist", orc[1]), ("E_hist", orc[2]), ("ee_hist", orc[3])):
            assert np.isfinite(f[name]).all()
            err = O.rel_err(f[name], o)
            assert err < bar_f, (label, name, err)
            record_error(f"{tag} {label} {name}", err, bar_f)
            diffs[(label, name)] = float(np.max(np.abs(f[name].astype(np.float64) - ref_f[name])))
        for name, a, o, r in (("g_f_iv", gfiv, o_gfiv, ref_gfiv), ("g_H", gH, o_gH, ref_gH)):
            err = O.rel_err(a, o)
            assert err < bar_g, (label, name, err)
            record_error(f"{tag} {label} {name}", err, bar_g)
            diffs[(label, name)] = float(np.max(np.abs(a.astype(np.float64) - r)))
        diffs[(label, "ee (vjp forward)")] = float(np.max(np.abs(ee_vjp.astype(np.float64) - ref_f["ee_hist"])))
    return diffs


@pytest.mark.parametrize("case", CASES, ids=["c2-grid", "shift2-f32", "shift2-f64"])
def test_slab_loops_equal_one_grid_path_bitwise(case, record_error):
    rings = [(f"{n} slabs", LocalRing(n)) for n in case[6]]
    diffs = _check_case(case, rings, record_error)
    bad = {k: v for k, v in diffs.items() if v != 0.0}
    assert not bad, f"slab results differ from the one-grid per-column path: {bad}"


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def test_dist_ring_one_rank_nccl(record_error):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", torch.cuda.current_device()))
    try:
        diffs = _check_case(CASES[1], [("dist 1 rank", DistRing())], record_error)
    finally:
        dist.destroy_process_group()
    bad = {k: v for k, v in diffs.items() if v != 0.0}
    assert not bad, f"slab results differ from the one-grid per-column path: {bad}"


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_plan_from_one_row_equals_plan_from_the_full_array(dtype):
    """vp_plan_create_from_row (f_eq as its nv-value row) gives the plan vp_plan_create gives for
    the broadcast (nx, nv) array: the same path and the same results bit for bit."""
    length_x, nx, nv, dt, T = CASES[0][:5]
    m, f_eq, f_iv, H, gEh, gff = _problem(length_x, nx, nv, dt, 12)
    full = Plan(m, dt, np.broadcast_to(f_eq, (nx, nv)), dtype=dtype)
    row = Plan(m, dt, f_eq, dtype=dtype)
    assert row.row_only and not full.row_only
    assert row.get_config() == full.get_config()
    a = full.forward(f_iv, H, 12, record_history=True)
    b = row.forward(f_iv, H, 12, record_history=True)
    torch.cuda.synchronize()
    for k in ("f_final", "f_hist", "E_hist", "ee_hist"):
        assert torch.equal(a[k], b[k]), k
