"""The forward entry point that allocates nothing, checked against the regular one.

``vp_forward_noalloc`` exists for callers that cannot allocate device memory when they run the
solver, for example code that must not call cudaMalloc (or go through an allocator) while it is
being captured into a CUDA graph, or a host application that owns all device memory. Its
scratch is one static device array of ``VP_NOALLOC_SCRATCH_BYTES`` (8 MiB) that every call
shares. This test calls it twice in a row through the C ABI, with different inputs, and checks
each result against ``vp_forward`` (which takes a caller-provided workspace) on the same inputs.
The second call checks that nothing left in the shared scratch by the first call leaks into it.
It also checks that a grid too large for the static scratch is refused with a clear error.

This file is named so that pytest collects it last.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

import vp_oracle as O
from conftest import two_stream_state
from warp_vp_solver_b200 import WarpVlasovPoissonSolver, _capi, make_mesh

pytestmark = pytest.mark.gpu


def _stream():
    return torch.cuda.current_stream().cuda_stream


def _run(lib, plan, f_iv, H, T, noalloc):
    nx, nv = plan.nx, plan.nv
    dev = plan.device
    f_final = torch.empty((nx, nv), dtype=torch.float64, device=dev)
    f_hist = torch.empty((T, nx, nv), dtype=plan.dtype, device=dev)
    E_hist = torch.empty((T, nx), dtype=plan.dtype, device=dev)
    ee_hist = torch.empty((T,), dtype=plan.dtype, device=dev)
    # fill the outputs with garbage so that unwritten entries would show
    for t in (f_final, f_hist, E_hist, ee_hist):
        t.fill_(float("nan"))
    if noalloc:
        rc = lib.vp_forward_noalloc(plan.handle, f_iv.data_ptr(), H.data_ptr(), T,
                                    f_final.data_ptr(), f_hist.data_ptr(), E_hist.data_ptr(),
                                    ee_hist.data_ptr(), _stream())
    else:
        ws = plan.workspace(T, 1)
        rc = lib.vp_forward(plan.handle, f_iv.data_ptr(), H.data_ptr(), T, f_final.data_ptr(),
                            f_hist.data_ptr(), E_hist.data_ptr(), ee_hist.data_ptr(), None, 1,
                            ws.data_ptr(), ws.numel(), _stream())
    _capi.check(rc)
    torch.cuda.synchronize()
    return [t.double().cpu().numpy() for t in (f_final, f_hist, E_hist, ee_hist)]


def test_noalloc_forward_matches_forward_on_two_calls_in_a_row():
    lib = _capi.load()
    m = make_mesh(10.0 * np.pi, 6.0, 128, 128)
    f_eq, f_iv = two_stream_state(m)
    s = WarpVlasovPoissonSolver(m, 0.05, f_eq)
    plan = s.plan
    T = 40
    f_dev = torch.tensor(f_iv, dtype=torch.float64, device=plan.device)
    fields = [np.zeros(m.nx), 0.01 * np.random.default_rng(1).standard_normal(m.nx)]
    for H_np in fields:   # two calls in a row, different inputs
        H = torch.tensor(H_np, dtype=plan.dtype, device=plan.device)
        got = _run(lib, plan, f_dev, H, T, noalloc=True)
        ref = _run(lib, plan, f_dev, H, T, noalloc=False)
        for a, b in zip(got, ref):
            assert np.isfinite(a).all()
            # same kernels on the same inputs: within the float32 parity tolerance (1e-5)
            assert O.rel_err(a, b) <= 1e-5


def test_noalloc_rejects_grid_larger_than_static_scratch():
    lib = _capi.load()
    m = make_mesh(10.0 * np.pi, 6.0, 1024, 1024)
    f_eq, f_iv = two_stream_state(m)
    plan = WarpVlasovPoissonSolver(m, 0.05, f_eq).plan
    f_dev = torch.tensor(f_iv, dtype=torch.float64, device=plan.device)
    H = torch.zeros(m.nx, dtype=plan.dtype, device=plan.device)
    E_hist = torch.empty((2, m.nx), dtype=plan.dtype, device=plan.device)
    rc = lib.vp_forward_noalloc(plan.handle, f_dev.data_ptr(), H.data_ptr(), 2, None, None,
                                E_hist.data_ptr(), None, _stream())
    assert rc == _capi.VP_ERR_ARG
    msg = _capi.last_error()
    assert "static scratch" in msg and str(8 << 20) in msg
