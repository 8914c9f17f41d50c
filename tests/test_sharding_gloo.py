"""Ensemble sharding over two ranks (gloo, CPU): each rank advances its LPT shard of an uneven
ensemble with no exchange during the time loop, one gather at the end, and the gathered
energy histories equal a single process's."""

from __future__ import annotations

import os
import socket
import sys

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _instances():
    from warp_vp_solver_b200 import make_mesh
    from warp_vp_solver_b200.workloads import fourier_coefficients, fourier_field, two_stream
    rng = np.random.default_rng(5)
    out = []
    for i in range(7):
        m = make_mesh(10 * np.pi, 6.0, int(rng.choice([8, 16])), int(rng.choice([16, 32])))
        f_eq, f_iv = two_stream(m, mu=float(rng.uniform(2, 3)), eps=1e-2)
        H = fourier_field(fourier_coefficients(4, 1e-2, i), m.xs, 2 * np.pi / m.period_x)
        out.append((m, f_eq, f_iv, H))
    return out


def _solve(inst, T=6, dt=0.05):
    import vp_oracle as O
    m, f_eq, f_iv, H = inst
    return O.delta_forward(O.grid_from(m), dt, f_eq, f_iv, H, T)[3]


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from warp_vp_solver_b200.sharding import lpt_shards
    inst = _instances()
    shards = lpt_shards([m.nx * m.nv for m, *_ in inst], world)
    mine = {i: _solve(inst[i]) for i in shards[rank]}
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    if rank == 0:
        merged = {}
        for d in gathered:
            merged.update(d)
        q.put({k: v.tolist() for k, v in merged.items()})
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_shards_match_serial():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    inst = _instances()
    assert sorted(int(k) for k in got) == list(range(len(inst)))
    for i, x in enumerate(inst):
        np.testing.assert_array_equal(np.asarray(got[i]), _solve(x))
