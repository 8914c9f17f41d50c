"""The forward entry point that allocates nothing, checked bit for bit against the regular one.

Some callers of this library cannot allocate device memory at the moment they run the solver:
code recorded into a CUDA graph under a capture mode that forbids cudaMalloc, plug-ins whose host
application owns all device memory through its own pool, and time-critical loops that cannot
take the device-wide synchronisation a cudaMalloc may cause. ``vp_forward_noalloc`` serves them:
its scratch is one static device array of ``VP_NOALLOC_SCRATCH_BYTES`` (8 MiB) that every call
shares and that keeps the previous call's contents.

The scratch holds the two delta-f state planes, the row partial sums, the completion counter and
the field vectors of the per-step kernels (or the row sums, field slices, energy partials and grid
barrier of the persistent loop); the cluster-resident kernels keep their state in shared memory
and never touch it. So each case here forces a path that uses it (per-column kernel, staged
kernel, a grid whose Poisson tail is its own launch, the persistent loop) and asserts it. Each case makes
two calls in a row with different inputs, and a call on a different grid sits between the cases,
so leftovers in the shared scratch would change a result. Every result must equal, bit for bit,
the regular ``vp_forward`` on the same inputs with a workspace pre-filled with garbage bytes.

This file is named so that pytest collects it last.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import two_stream_state
from warp_vp_solver_b200 import WarpVlasovPoissonSolver, _capi, make_mesh

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 8 << 20

# (nx, nv, path): "column" = per-column kernel with the tail inside the step launch, "staged" =
# staged kernel, "staged_tail" = staged kernel with the Poisson tail as its own launch (nx > 2048),
# "persist" = one cooperative launch for the whole loop
CASES = [(128, 128, "column"), (128, 512, "staged"), (4096, 128, "staged_tail"), (128, 512, "persist")]


def _stream():
    return torch.cuda.current_stream().cuda_stream


def _solver(nx, nv, path):
    m = make_mesh(10.0 * np.pi, 6.0, nx, nv)
    f_eq, _ = two_stream_state(m)
    s = WarpVlasovPoissonSolver(m, 0.05, f_eq)
    if path == "column":
        s.plan.set_config(cluster_size=0, stage_rows=0, persist_rows=0)
    elif path == "persist":
        s.plan.set_config(cluster_size=0, persist_rows=4)
    else:
        s.plan.set_config(cluster_size=0, persist_rows=0)
    cfg = s.plan.get_config()
    assert cfg["cluster_size"] == 0, "the cluster-resident path would not use the scratch"
    assert (cfg["persist_rows"] > 0) == (path == "persist")
    assert (cfg["stage_rows"] > 0) == (path != "column")
    assert (cfg["tail_inline"] == 0) == (path == "staged_tail")
    return m, f_eq, s


def _inputs(m, f_eq, seed):
    rng = np.random.default_rng(seed)
    f_iv = (1.0 + 10 ** rng.uniform(-3, -2) * np.cos(0.2 * m.X + rng.uniform(0, 6))) * f_eq
    H = 0.02 * rng.standard_normal(m.nx)
    return f_iv, H


def _run(lib, plan, f_iv, H, T, noalloc):
    nx, nv, dev = plan.nx, plan.nv, plan.device
    f_final = torch.full((nx, nv), float("nan"), dtype=torch.float64, device=dev)
    f_hist = torch.full((T, nx, nv), float("nan"), dtype=plan.dtype, device=dev)
    E_hist = torch.full((T, nx), float("nan"), dtype=plan.dtype, device=dev)
    ee_hist = torch.full((T,), float("nan"), dtype=plan.dtype, device=dev)
    f_dev = torch.tensor(f_iv, dtype=torch.float64, device=dev)
    H_dev = torch.tensor(H, dtype=plan.dtype, device=dev)
    if noalloc:
        rc = lib.vp_forward_noalloc(plan.handle, f_dev.data_ptr(), H_dev.data_ptr(), T,
                                    f_final.data_ptr(), f_hist.data_ptr(), E_hist.data_ptr(),
                                    ee_hist.data_ptr(), _stream())
    else:
        ws = plan.workspace(T, 1)
        ws.view(torch.uint8).fill_(0xA5)   # garbage: the regular path must not rely on zeros
        rc = lib.vp_forward(plan.handle, f_dev.data_ptr(), H_dev.data_ptr(), T, f_final.data_ptr(),
                            f_hist.data_ptr(), E_hist.data_ptr(), ee_hist.data_ptr(), None, 1,
                            ws.data_ptr(), ws.numel() * ws.element_size(), _stream())
    _capi.check(rc)
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in (f_final, f_hist, E_hist, ee_hist)]


def test_noalloc_forward_equals_forward_bitwise_on_calls_in_a_row():
    lib = _capi.load()
    T = 12
    for case_no, (nx, nv, path) in enumerate(CASES):
        m, f_eq, s = _solver(nx, nv, path)
        assert s.plan.workspace_bytes(T, 1) <= SCRATCH_BYTES
        for call in range(2):   # two calls in a row, different inputs
            f_iv, H = _inputs(m, f_eq, seed=100 * case_no + call)
            got = _run(lib, s.plan, f_iv, H, T, noalloc=True)
            ref = _run(lib, s.plan, f_iv, H, T, noalloc=False)
            for name, a, b in zip(("f_final", "f_hist", "E_hist", "ee_hist"), got, ref):
                assert np.isfinite(a).all(), f"{nx}x{nv} {path} call {call}: {name} not written"
                assert np.array_equal(a, b), f"{nx}x{nv} {path} call {call}: {name} differs"


def test_noalloc_rejects_grids_larger_than_the_static_scratch():
    lib = _capi.load()
    for nx, nv, dtype, name in [(1024, 1024, torch.float32, "float32"),
                                (512, 1024, torch.float64, "float64")]:
        m = make_mesh(10.0 * np.pi, 6.0, nx, nv)
        f_eq, f_iv = two_stream_state(m)
        plan = WarpVlasovPoissonSolver(m, 0.05, f_eq, dtype=dtype).plan
        assert plan.workspace_bytes(2, 1) > SCRATCH_BYTES
        f_dev = torch.tensor(f_iv, dtype=torch.float64, device=plan.device)
        H = torch.zeros(m.nx, dtype=plan.dtype, device=plan.device)
        E_hist = torch.empty((2, m.nx), dtype=plan.dtype, device=plan.device)
        rc = lib.vp_forward_noalloc(plan.handle, f_dev.data_ptr(), H.data_ptr(), 2, None, None,
                                    E_hist.data_ptr(), None, _stream())
        assert rc == _capi.VP_ERR_ARG
        msg = _capi.last_error()
        assert "static scratch" in msg and str(SCRATCH_BYTES) in msg and name in msg
