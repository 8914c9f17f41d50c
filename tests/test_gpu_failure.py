"""Failure detection on the device, without faulting, trapping or hanging the GPU.

* Non-finite inputs that live on the device: ``vp_forward`` never synchronises, so it cannot
  return an error for values it has not looked at; a check kernel at the start of the call raises
  VP_STATUS_NONFINITE_INPUT in the plan's status word instead, and ``check_status`` reports it.
* Bounded waits: the tensor-core MLP kernels wait on mbarriers with a limit. With the limit set
  to zero a wait is one non-blocking test of the barrier, and the warps that do not issue MMAs
  reach it before the issuing thread has committed them, so it gives up: the status flag must be
  raised, the call must return normally (after draining its own MMAs) and the CUDA context must
  stay usable: with the default limit restored, the same network computes the same outputs.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import two_stream_state
from warp_vp_solver_b200 import WarpVlasovPoissonSolver, make_mesh
from warp_vp_solver_b200.mlp import MLP

pytestmark = pytest.mark.gpu


def test_device_non_finite_input_raises_status_flag():
    m = make_mesh(10.0 * np.pi, 6.0, 64, 64)
    f_eq, f_iv = two_stream_state(m)
    s = WarpVlasovPoissonSolver(m, 0.05, f_eq)
    s.check_status()   # clean
    f = torch.tensor(f_iv, device="cuda")
    H = torch.zeros(m.nx, device="cuda")
    s.run_forward(f, H, 0.5)
    s.check_status()   # finite inputs raise nothing
    f_bad = f.clone()
    f_bad[7, 9] = float("nan")
    s.run_forward(f_bad, H, 0.5)   # returns without synchronising
    with pytest.raises(ValueError, match="NaN or infinite"):
        s.check_status()
    s.check_status()   # the check cleared the flag
    H_bad = H.clone()
    H_bad[3] = float("inf")
    s.run_forward(f, H_bad, 0.5)
    assert s.plan.status() & 1
    s.plan.clear_status()
    assert s.plan.status() == 0


def test_mlp_zero_wait_limit_raises_flag_and_returns_cleanly():
    net = MLP([32, 256, 256, 100], max_batch=512, seed=3)
    X = torch.randn(512, 32, device="cuda")
    ref = net.forward(X).clone()
    torch.cuda.synchronize()
    assert net.status() == 0
    net.set_wait_limit(0)
    out = net.forward(X)     # every GEMM CTA gives up at its first poll, drains and returns
    torch.cuda.synchronize()
    assert net.status() & 1
    assert out.shape == ref.shape
    net.set_wait_limit(1_000_000_000)
    net.clear_status()
    again = net.forward(X)
    torch.cuda.synchronize()
    assert net.status() == 0
    assert torch.equal(again, ref)
