"""The persistent forward loop (one cooperative launch per forward loop, vp_persist.cu) against the
float64 delta-f oracle, the staged per-step kernels and itself.

It covers both ways the kernel solves the field (every CTA on its own window rows, or slices plus
a second grid barrier), band heights 4, 8 and 16 (one or several bands per CTA), fields strong
enough to shift rows by several cells (the table and the far-shift forms of the v step), the
adjoint's recomputation of checkpoint segments by the same kernel, and the bounded grid barrier.

Bars (max-norm relative error): float32 forward 1e-5 and adjoint 5e-5 against the oracle (the
largest adjoint error measured on B200 is 3.2e-6, with fields that shift rows by several cells).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import vp_oracle as O
from conftest import two_stream_state
from warp_vp_solver_b200 import WarpVlasovPoissonSolver, make_mesh
from warp_vp_solver_b200.workloads import bump_on_tail

pytestmark = pytest.mark.gpu

FIELDS = ("f_final", "f_hist", "E_hist", "ee_hist")


def _solver(m, dt, f_eq, rows=None, **kw):
    s = WarpVlasovPoissonSolver(m, dt, f_eq, **kw)
    s.plan.set_config(cluster_size=0, persist_rows=rows if rows is not None else 4)
    cfg = s.plan.get_config()
    assert cfg["persist_rows"] > 0 and cfg["persist_ctas"] > 0
    return s


# (nx, nv, set-up, field amplitude, band rows): two-stream and bump-on-tail, weak to strong fields
SHAPES = [
    (64, 256, "two_stream", 0.02, 4),
    (128, 512, "two_stream", 0.3, 8),
    (128, 512, "two_stream", 2.0, 16),    # shifts beyond the 4-cell staged halo
    (64, 512, "bump_on_tail", 0.05, 4),
    (4096, 512, "two_stream", 0.05, 16),  # field solved in slices (second grid barrier)
]


def _setup(nx, nv, kind, amp):
    if kind == "two_stream":
        m = make_mesh(10.0 * np.pi, 6.0, nx, nv)
        f_eq, f_iv = two_stream_state(m, eps=1e-2)
    else:
        m = make_mesh(2.0 * np.pi / 0.3, 8.0, nx, nv)
        f_eq, f_iv = bump_on_tail(m)
    H = amp * np.random.default_rng(nx + nv).standard_normal(nx)
    return m, f_eq, f_iv, H


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: f"{s[0]}x{s[1]}_{s[2]}_H{s[3]}_R{s[4]}")
def test_persistent_forward_and_adjoint_match_oracle(shape, record_error):
    nx, nv, kind, amp, rows = shape
    m, f_eq, f_iv, H = _setup(nx, nv, kind, amp)
    T, dt = 6, 0.05
    s = _solver(m, dt, f_eq, rows, checkpoint_every=3)
    out = s.run_forward(f_iv, H, T * dt)
    g = O.grid_from(m)
    ref = O.delta_forward(g, dt, f_eq, f_iv, H, T)
    worst = 0.0
    for arr, r, name in zip(out, ref, FIELDS):
        err = O.rel_err(arr, r)
        worst = max(worst, err)
        assert err < 1e-5, f"{name}: {err:.2e}"
    record_error(f"persist {nx}x{nv} {kind} H{amp} R{rows} fwd", worst, 1e-5)
    if nx > 1024:
        return   # the float64 oracle's adjoint at this size is slow; the forward was the point
    w = O.trapezoid_time_weights(T, dt)
    rg = np.random.default_rng(3)
    gff = rg.standard_normal((nx, nv))
    gfh = 0.1 * rg.standard_normal((T, nx, nv))
    gEh = rg.standard_normal((T, nx))
    gf, gH = s._run_backward(f_iv, H, T * dt, None, gff, gfh, gEh, w)
    rf, rH = O.delta_backward(g, dt, f_eq, f_iv, H, T, gff, gfh, gEh, w)
    e = max(O.rel_err(gf, rf), O.rel_err(gH, rH))
    record_error(f"persist {nx}x{nv} {kind} H{amp} R{rows} adj", e, 5e-5)
    assert e < 5e-5, f"adjoint {e:.2e}"


def test_checkpoint_recompute_by_the_persistent_kernel_is_bitwise_neutral():
    """The adjoint recomputes checkpoint segments with the forward's own kernel (replay mode), so
    the gradient does not depend on the checkpoint interval by a single bit."""
    m, f_eq, f_iv, H = _setup(128, 512, "two_stream", 0.3)
    T, dt = 9, 0.05
    w = O.trapezoid_time_weights(T, dt)
    outs = []
    for every in (1, 2, 4, 0):
        s = _solver(m, dt, f_eq, 8, checkpoint_every=every or None)
        outs.append(s._run_backward(f_iv, H, T * dt, None, None, None, None, w))
    for gf, gH in outs[1:]:
        assert np.array_equal(gf, outs[0][0]) and np.array_equal(gH, outs[0][1])


def test_persistent_agrees_with_staged_kernels_and_is_deterministic():
    m, f_eq, f_iv, H = _setup(128, 512, "two_stream", 0.3)
    T, dt = 8, 0.05
    s = _solver(m, dt, f_eq, 4)
    a = s.run_forward(f_iv, H, T * dt)
    b = s.run_forward(f_iv, H, T * dt)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    st = WarpVlasovPoissonSolver(m, dt, f_eq)
    st.plan.set_config(cluster_size=0, persist_rows=0)
    assert st.plan.get_config()["stage_rows"] > 0
    c = st.run_forward(f_iv, H, T * dt)
    for x, y, name in zip(a, c, FIELDS):
        assert O.rel_err(x, y) < 2e-6, name


def test_plan_default_paths_by_grid_size():
    """Configuration 3's grid runs the persistent loop by default; a cluster-resident grid keeps
    its one-cluster kernels; a 4096-row grid (field solved in slices) runs the strip step kernels
    unless persist_rows asks for the persistent loop."""
    def plan(lx, lv, nx, nv):
        m = make_mesh(lx, lv, nx, nv)
        return WarpVlasovPoissonSolver(m, 0.05, np.ones((nx, nv)) * np.exp(-0.5 * m.vs ** 2)[None, :]).plan
    cfg = plan(2 * np.pi / 0.3, 8.0, 512, 1024).get_config()
    assert cfg["cluster_size"] == 0 and cfg["persist_rows"] > 0, cfg
    p = plan(10.0 * np.pi, 6.0, 256, 256)
    assert p.get_config()["cluster_size"] > 0 and p.get_config()["persist_rows"] == 0
    q = plan(10.0 * np.pi, 6.0, 4096, 1024)   # field in slices: strip step kernels by default
    assert q.get_config()["persist_rows"] == 0 and q.get_config()["strip_rows"] == 4
    q.set_config(persist_rows=16, strip_rows=0)
    assert q.get_config()["persist_rows"] == 16 and q.get_config()["strip_rows"] == 0


def test_grid_barrier_wait_limit_zero_times_out_cleanly():
    """With a zero wait limit every CTA but the last to arrive gives up at the first grid
    barrier: the launch ends early with VP_STATUS_WAIT_TIMEOUT raised, and the context stays
    usable (with the default limit restored the same call gives the normal result)."""
    m, f_eq, f_iv, H = _setup(128, 512, "two_stream", 0.05)
    T, dt = 5, 0.05
    s = _solver(m, dt, f_eq, 4)
    assert s.plan.get_config()["persist_ctas"] >= 2
    ref = s.run_forward(f_iv, H, T * dt)
    s.check_status()
    s.plan.set_wait_limit(0)
    s.run_forward(f_iv, H, T * dt)
    torch.cuda.synchronize()
    assert s.plan.status() & 2
    with pytest.raises(RuntimeError, match="wait ran out"):
        s.check_status()
    s.plan.set_wait_limit(1_000_000_000)
    again = s.run_forward(f_iv, H, T * dt)
    s.check_status()
    for x, y in zip(ref, again):
        assert np.array_equal(x, y)
