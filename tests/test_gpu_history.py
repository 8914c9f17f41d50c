"""f_hist streamed to pinned host memory through a device ring (vp_forward_stream_history) is
bitwise the history the device path records, for the Strang and merged schemes, with ring reuse
and checkpointing; numpy callers get it through run_forward."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import two_stream_state
from warp_vp_solver_b200 import WarpVlasovPoissonSolver, make_mesh

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("merged", [False, True])
@pytest.mark.parametrize("slots,every", [(2, 1), (3, 4), (8, 0)])
def test_streamed_history_equals_device_history(merged, slots, every):
    m = make_mesh(10.0 * np.pi, 6.0, 64, 256)
    f_eq, f_iv = two_stream_state(m, eps=1e-2)
    H = 0.05 * np.random.default_rng(0).standard_normal(m.nx)
    s = WarpVlasovPoissonSolver(m, 0.05, f_eq, aggressive=merged, checkpoint_every=every or None)
    s.plan.set_config(cluster_size=0, persist_rows=0)
    T = 11
    dev = s.plan.forward(f_iv, H, T, record_history=True)
    st = s.plan.forward_stream_history(f_iv, H, T, slots=slots, want_tape=True)
    torch.cuda.synchronize()
    assert st["f_hist"].is_pinned()
    assert torch.equal(st["f_hist"], dev["f_hist"].cpu())
    assert torch.equal(st["f_final"], dev["f_final"])
    assert torch.equal(st["ee_hist"], dev["ee_hist"])


def test_run_forward_streams_when_asked():
    m = make_mesh(10.0 * np.pi, 6.0, 32, 128)
    f_eq, f_iv = two_stream_state(m, eps=1e-2)
    H = np.zeros(m.nx)
    a = WarpVlasovPoissonSolver(m, 0.05, f_eq)
    a.history_on_host = True
    b = WarpVlasovPoissonSolver(m, 0.05, f_eq)
    b.history_on_host = False
    b.plan.set_config(cluster_size=0)
    ra = a.run_forward(f_iv, H, 0.4)
    rb = b.run_forward(f_iv, H, 0.4)
    for x, y in zip(ra, rb):
        np.testing.assert_array_equal(x, y)
