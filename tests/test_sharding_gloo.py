"""Ensemble sharding over two ranks (gloo, CPU) through the product's host path,
``sharding.solve_sharded_ensemble``: each rank solves its longest-processing-time share of an
uneven ensemble with no exchange during the time loops, one all_gather brings every instance's
energy history, field history and dJ/dH to every rank, and the result equals a single process's.
The per-shard solve is injected (the float64 oracle on CPU); on a GPU the default solves the
shard as one Ensemble (tests/test_gpu_ensemble.py)."""

from __future__ import annotations

import os
import socket
import sys

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
T_STEPS = 6


def _instances():
    from warp_vp_solver_b200 import make_mesh
    from warp_vp_solver_b200.workloads import fourier_coefficients, fourier_field, two_stream
    rng = np.random.default_rng(5)
    meshes, dts, feqs, fivs, Hs = [], [], [], [], []
    for i in range(7):
        m = make_mesh(10 * np.pi, 6.0, int(rng.choice([8, 16])), int(rng.choice([16, 32])))
        f_eq, f_iv = two_stream(m, mu=float(rng.uniform(2, 3)), eps=1e-2)
        meshes.append(m)
        dts.append(float(rng.choice([0.05, 0.04])))
        feqs.append(f_eq)
        fivs.append(f_iv)
        Hs.append(fourier_field(fourier_coefficients(4, 1e-2, i), m.xs, 2 * np.pi / m.period_x))
    return meshes, dts, feqs, fivs, Hs


def oracle_shard(meshes, dts, f_eqs, f_ivs, Hs, n_steps, want_grad):
    """The per-shard solve on CPU: the float64 delta-f oracle, instance by instance."""
    import vp_oracle as O
    out = []
    for m, dt, f_eq, f_iv, H in zip(meshes, dts, f_eqs, f_ivs, Hs):
        g = O.grid_from(m)
        fwd = O.delta_forward(g, float(dt), f_eq, f_iv, H, n_steps)
        rec = {"ee_hist": fwd[3], "E_hist": fwd[2]}
        if want_grad:
            w = O.trapezoid_time_weights(n_steps, float(dt))
            rec["g_H"] = O.delta_backward(g, float(dt), f_eq, f_iv, H, n_steps, np.zeros((m.nx, m.nv)),
                                          None, np.zeros((n_steps, m.nx)), w)[1]
        out.append(rec)
    return out


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from test_sharding_gloo import _instances, oracle_shard
    from warp_vp_solver_b200.sharding import lpt_shards, solve_sharded_ensemble
    meshes, dts, feqs, fivs, Hs = _instances()
    calls = []

    def counting(*a):
        calls.append(len(a[0]))
        return oracle_shard(*a)

    res = solve_sharded_ensemble(meshes, dts, feqs, fivs, Hs, T_STEPS, want_grad=True, solve_shard=counting)
    shards = lpt_shards([m.nx * m.nv for m in meshes], world)
    q.put({"rank": rank, "solved": calls, "expected": len(shards[rank]),
           "res": [{k: v.tolist() for k, v in r.items()} for r in res]})
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharded_ensemble_matches_serial():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    outs = [q.get(timeout=180) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    meshes, dts, feqs, fivs, Hs = _instances()
    serial = oracle_shard(meshes, dts, feqs, fivs, Hs, T_STEPS, True)
    for o in outs:
        # each rank solved only its own share, and both shares together are the ensemble
        assert o["solved"] == [o["expected"]] and 0 < o["expected"] < len(meshes)
        assert len(o["res"]) == len(meshes)
        for got, ref in zip(o["res"], serial):
            for k in ("ee_hist", "E_hist", "g_H"):
                np.testing.assert_array_equal(np.asarray(got[k]), ref[k])
    assert sum(o["expected"] for o in outs) == len(meshes)


def test_single_process_sharded_ensemble_is_a_plain_solve():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from warp_vp_solver_b200.sharding import solve_sharded_ensemble
    meshes, dts, feqs, fivs, Hs = _instances()
    res = solve_sharded_ensemble(meshes, dts, feqs, fivs, Hs, T_STEPS, want_grad=False,
                                 solve_shard=oracle_shard)
    ref = oracle_shard(meshes, dts, feqs, fivs, Hs, T_STEPS, False)
    for got, r in zip(res, ref):
        assert set(got) == {"ee_hist", "E_hist"}
        np.testing.assert_array_equal(got["ee_hist"], r["ee_hist"])
