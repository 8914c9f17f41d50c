"""x-slab decomposition: the product's host loop (``slab.SlabSolver``) on CPU.

The per-slab calls are the float64 CPU restatement (``oracle/vp_slab_oracle.py``), injected in
place of the CUDA ones; what runs is the product's orchestration: ghost-row exchanges, row-sum
gathers, the replicated field solve and the checkpointed adjoint's segment replays. Results are
compared with the whole-grid float64 delta oracle (``vp_oracle.delta_forward`` /
``delta_backward``). ``LocalRing`` holds every slab in one process; ``DistRing`` runs one slab per
gloo rank (two and three spawned processes)."""

from __future__ import annotations

import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import vp_oracle as O
from vp_slab_oracle import OracleSlabOps
from warp_vp_solver_b200.slab import DistRing, LocalRing, SlabSolver, slab_bounds

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# (length_x, nx, nv, dt, T): the second case shifts columns by up to 4 cells per half step
CASES = [(10 * np.pi, 24, 32, 0.05, 7), (2 * np.pi, 64, 32, 0.2, 9)]


def _problem(length_x, nx, nv, dt, T, seed=0):
    from warp_vp_solver_b200 import make_mesh
    m = make_mesh(length_x, 6.0, nx, nv)
    g = O.grid_from(m)
    f_eq = (np.exp(-0.5 * (m.vs - 2.4) ** 2) + np.exp(-0.5 * (m.vs + 2.4) ** 2)) / (2 * np.sqrt(2 * np.pi))
    rng = np.random.default_rng(seed)
    f_iv = (1.0 + 1e-2 * np.cos(2 * np.pi / length_x * m.X) + 1e-3 * rng.standard_normal((nx, nv))) * f_eq[None, :]
    H = 0.05 * rng.standard_normal(nx)
    gEh = 1e-2 * rng.standard_normal((T, nx))
    gff = 1e-1 * rng.standard_normal((nx, nv))
    return m, g, f_eq, f_iv, H, gEh, gff


def _solver(m, g, f_eq, dt, ring):
    return SlabSolver(m, dt, f_eq, ring, dtype=torch.float64,
                      ops_factory=lambda r0, n: OracleSlabOps(g, dt, f_eq, r0, n))


def _rows(a, bounds, local):
    return {s: a[bounds[s][0]:bounds[s][0] + bounds[s][1]] for s in local}


def _join(parts, bounds):
    return np.concatenate([np.asarray(parts[s]) for s in range(len(bounds))])


def test_slab_bounds():
    assert slab_bounds(10, 3) == [(0, 3), (3, 3), (6, 4)]
    assert slab_bounds(8, 1) == [(0, 8)]
    with pytest.raises(ValueError):
        slab_bounds(4, 5)


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("n_slabs", [1, 2, 3])
def test_local_ring_matches_whole_grid_oracle(case, n_slabs):
    length_x, nx, nv, dt, T = case
    m, g, f_eq, f_iv, H, gEh, gff = _problem(*case)
    s = _solver(m, g, f_eq, dt, LocalRing(n_slabs))
    b = s.bounds
    ff, fh, Eh, eeh = s.run_forward(_rows(f_iv, b, s.ring.local), H, T * dt, record_history=True)
    ref = O.delta_forward(g, dt, np.broadcast_to(f_eq, (nx, nv)), f_iv, H, T)
    assert O.rel_err(_join(ff, b), ref[0]) < 1e-12
    assert O.rel_err(np.concatenate([fh[k].numpy() for k in range(n_slabs)], axis=1), ref[1]) < 1e-12
    assert O.rel_err(Eh.numpy(), ref[2]) < 1e-12
    assert O.rel_err(eeh.numpy(), ref[3]) < 1e-12

    w = O.trapezoid_time_weights(T, dt)
    for K in (None, 1, 3):
        out = s.vjp(_rows(f_iv, b, s.ring.local), H, T * dt, g_E_hist=gEh, g_ee_hist=w,
                    g_f_final_rows=_rows(gff, b, s.ring.local), checkpoint_every=K)
        g_fiv, g_H = O.delta_backward(g, dt, np.broadcast_to(f_eq, (nx, nv)), f_iv, H, T, gff, None, gEh, w)
        assert O.rel_err(out["g_H"].numpy(), g_H) < 1e-11, K
        assert O.rel_err(_join({k: v.numpy() for k, v in out["g_f_iv"].items()}, b), g_fiv) < 1e-11, K


def test_slabs_thinner_than_the_ghost_rows_are_refused():
    m, g, f_eq, *_ = _problem(*CASES[1])
    with pytest.raises(ValueError, match="ghost rows"):
        _solver(m, g, f_eq, CASES[1][3], LocalRing(16))


def _worker(rank, world, port, case, q):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        length_x, nx, nv, dt, T = case
        m, g, f_eq, f_iv, H, gEh, gff = _problem(*case)
        s = _solver(m, g, f_eq, dt, DistRing())
        b = s.bounds
        ff, _, Eh, eeh = s.run_forward(_rows(f_iv, b, [rank]), H, T * dt)
        w = O.trapezoid_time_weights(T, dt)
        out = s.vjp(_rows(f_iv, b, [rank]), H, T * dt, g_E_hist=gEh, g_ee_hist=w,
                    g_f_final_rows=_rows(gff, b, [rank]))
        q.put((rank, ff[rank].numpy(), Eh.numpy(), eeh.numpy(), out["g_H"].numpy(), out["g_f_iv"][rank].numpy()))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_dist_ring_on_gloo_ranks_matches_whole_grid_oracle(world):
    case = CASES[1]
    length_x, nx, nv, dt, T = case
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, case, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        r = q.get(timeout=240)
        res[r[0]] = r
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    m, g, f_eq, f_iv, H, gEh, gff = _problem(*case)
    feq2 = np.broadcast_to(f_eq, (nx, nv))
    ref = O.delta_forward(g, dt, feq2, f_iv, H, T)
    w = O.trapezoid_time_weights(T, dt)
    g_fiv, g_H = O.delta_backward(g, dt, feq2, f_iv, H, T, gff, None, gEh, w)
    assert O.rel_err(np.concatenate([res[r][1] for r in range(world)]), ref[0]) < 1e-12
    assert O.rel_err(np.concatenate([res[r][5] for r in range(world)]), g_fiv) < 1e-11
    for r in range(world):
        assert O.rel_err(res[r][2], ref[2]) < 1e-12
        assert O.rel_err(res[r][3], ref[3]) < 1e-12
        assert O.rel_err(res[r][4], g_H) < 1e-11


def test_slab_abi_rejects_null_handles_without_a_device():
    import ctypes
    from warp_vp_solver_b200 import _capi
    lib = _capi.load()
    out = ctypes.c_void_p()
    assert lib.vp_slab_create(None, 0, 4, ctypes.byref(out)) == _capi.VP_ERR_ARG
    assert "must not be NULL" in _capi.last_error()
    assert lib.vp_slab_forward_start(None, None, None, None, None) == _capi.VP_ERR_ARG
    assert lib.vp_slab_backward_finish(None, None, None, None, None, None) == _capi.VP_ERR_ARG
    assert lib.vp_slab_destroy(None) == 0


def test_plan_from_row_rejects_null_arguments_without_a_device():
    import ctypes
    from warp_vp_solver_b200 import _capi
    lib = _capi.load()
    out = ctypes.c_void_p()
    assert lib.vp_plan_create_from_row(None, 0.1, None, 0, ctypes.byref(out)) == _capi.VP_ERR_ARG
    assert "must not be NULL" in _capi.last_error()
