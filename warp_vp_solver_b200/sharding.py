"""Ensemble sharding across ranks (one process per GPU).

Instances are independent, so an ensemble splits across ranks with no data-path collective:
longest-processing-time-first assignment of instance costs (cells per step) to the currently
lightest rank. Every rank computes the same assignment from the same costs, so no exchange is
needed to agree on it. ``solve_sharded_ensemble`` runs a rank's share and gathers every
instance's results with one collective.
"""

from __future__ import annotations

import heapq
from typing import Callable, Sequence

import numpy as np
import torch


def lpt_shards(costs: Sequence[float], n_ranks: int) -> list[list[int]]:
    """Instance indices per rank (each list ascending). Deterministic: ties go to the lower rank."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(n_ranks)]
    heapq.heapify(heap)
    shards: list[list[int]] = [[] for _ in range(n_ranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(s) for s in shards]


def shard_loads(costs: Sequence[float], shards: list[list[int]]) -> list[float]:
    return [float(sum(costs[i] for i in s)) for s in shards]


def _trapezoid_weights(n: int, dt: float) -> np.ndarray:
    """dJ/dee for J = trapezoid(ee, dx=dt) (warp_vp_solver/utils.py:111-116)."""
    w = np.full(n, float(dt))
    if n >= 1:
        w[0] *= 0.5
        w[-1] *= 0.5
    if n == 1:
        w[0] = 0.0
    return w


def solve_shard_on_device(meshes, dts, f_eqs, f_ivs, Hs, n_steps: int, want_grad: bool = True,
                          dtype=torch.float32, device=None) -> list[dict]:
    """Forward (and the adjoint of J_i = trapezoid(ee_i, dt_i)) of a list of instances as one
    :class:`~warp_vp_solver_b200.ensemble.Ensemble` on this rank's device; per instance a dict of
    NumPy float64 arrays ``ee_hist`` (T), ``E_hist`` (T, nx) and, with ``want_grad``, ``g_H`` (nx)."""
    from .ensemble import Ensemble
    if not meshes:
        return []
    ens = Ensemble(meshes, dts, f_eqs, dtype=dtype, device=device)
    H = ens.pack_rows(Hs)
    out = ens.forward(ens.pack_cells(f_ivs), H, n_steps, want_tape=want_grad, want_f_final=False)
    res = [{"ee_hist": ens.ee_of(out["ee_hist"], i, n_steps).double().cpu().numpy(),
            "E_hist": ens.hist_of(out["E_hist"], i, n_steps).double().cpu().numpy()} for i in range(ens.n)]
    if want_grad:
        w = np.concatenate([_trapezoid_weights(n_steps, float(np.broadcast_to(dts, (ens.n,))[i]))
                            for i in range(ens.n)])
        g_ee = torch.tensor(w, dtype=ens.dtype, device=ens.device)
        _, g_H = ens.backward(H, n_steps, out["tape"], g_ee_hist=g_ee)
        for i in range(ens.n):
            res[i]["g_H"] = ens.rows_of(g_H, i).double().cpu().numpy()
    ens.close()
    return res


def solve_sharded_ensemble(meshes: Sequence, dts, f_eqs: Sequence, f_ivs: Sequence, Hs: Sequence,
                           n_steps: int, want_grad: bool = True, group=None,
                           solve_shard: Callable | None = None) -> list[dict]:
    """Solve an ensemble of independent instances split over the ranks of a process group.

    Every rank passes the FULL instance list and gets back every instance's results, in the
    caller's order. Rank r solves ``lpt_shards(nx*nv costs, world)[r]`` (the same assignment on
    every rank, no exchange needed) with ``solve_shard(meshes, dts, f_eqs, f_ivs, Hs, n_steps,
    want_grad) -> list of dicts`` (default: one :class:`Ensemble` on this rank's CUDA device,
    :func:`solve_shard_on_device`); nothing is exchanged while the time loops run. The results
    (``ee_hist`` (T), ``E_hist`` (T, nx) and, with ``want_grad``, ``g_H`` = dJ_i/dH_i for
    J_i = trapezoid(ee_i, dt_i)) are then packed into one float64 buffer per rank in a layout
    every rank can compute, and gathered with ONE ``all_gather``. Without an initialised process
    group this is a single-rank solve. The reference advances one solver at a time
    (warp_vp_solver/solver.py:418-612); it has no multi-device path.
    """
    import torch.distributed as dist

    n = len(meshes)
    dts = np.broadcast_to(np.asarray(dts, dtype=np.float64), (n,))
    distributed = dist.is_available() and dist.is_initialized()
    rank = dist.get_rank(group) if distributed else 0
    world = dist.get_world_size(group) if distributed else 1
    solve = solve_shard or solve_shard_on_device
    shards = lpt_shards([int(m.nx) * int(m.nv) for m in meshes], world)
    mine = shards[rank]
    local = solve([meshes[i] for i in mine], dts[mine], [f_eqs[i] for i in mine], [f_ivs[i] for i in mine],
                  [Hs[i] for i in mine], n_steps, want_grad)
    if len(local) != len(mine):
        raise RuntimeError(f"solve_shard returned {len(local)} results for {len(mine)} instances")
    fields = ["ee_hist", "E_hist"] + (["g_H"] if want_grad else [])

    def size_of(i):
        nx = int(meshes[i].nx)
        return n_steps + n_steps * nx + (nx if want_grad else 0)

    if world == 1:
        return [{k: np.asarray(local[p][k], dtype=np.float64) for k in fields} for p in range(len(mine))]
    sizes = [sum(size_of(i) for i in s) for s in shards]
    width = max(max(sizes), 1)
    buf = np.zeros(width)
    off = 0
    for p, i in enumerate(mine):
        for k in fields:
            a = np.asarray(local[p][k], dtype=np.float64).reshape(-1)
            buf[off:off + a.size] = a
            off += a.size
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    mine_t = torch.as_tensor(buf, device=dev)
    parts = [torch.empty(width, dtype=torch.float64, device=dev) for _ in range(world)]
    dist.all_gather(parts, mine_t, group=group)
    results: list[dict | None] = [None] * n
    for r, s in enumerate(shards):
        flat = parts[r].cpu().numpy()
        off = 0
        for i in s:
            nx = int(meshes[i].nx)
            shapes = {"ee_hist": (n_steps,), "E_hist": (n_steps, nx), "g_H": (nx,)}
            rec = {}
            for k in fields:
                cnt = int(np.prod(shapes[k]))
                rec[k] = flat[off:off + cnt].reshape(shapes[k]).copy()
                off += cnt
            results[i] = rec
    return results
