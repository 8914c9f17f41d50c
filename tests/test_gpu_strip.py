"""The strip step kernels (vp_strip.cu: a strip kernel and a circulant field kernel per step, for
large grids) against the float64 delta-f oracle, the persistent loop and themselves.

It covers band heights 4, 8 and 16, runs of bands that cross a chunk boundary (grids whose tile count
is not a multiple of the CTA count), fields strong enough to shift rows by several cells (the table
and far-shift forms of the v step, V^T and the slope), the adjoint's recomputation of checkpoint
segments by the same kernel, and the f_hist / f_final outputs.

Bars (max-norm relative error): float32 forward 1e-5 and adjoint 5e-5 against the oracle, as for
the persistent loop (same tile arithmetic, field by the same circulant).
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


def _solver(m, dt, f_eq, rows, cols=256, **kw):
    s = WarpVlasovPoissonSolver(m, dt, f_eq, **kw)
    s.plan.set_config(cluster_size=0, persist_rows=0, strip_rows=rows, strip_cols=cols)
    cfg = s.plan.get_config()
    assert cfg["strip_rows"] == rows and cfg["strip_ctas"] > 0 and cfg["persist_rows"] == 0
    assert cfg["strip_cols"] == cols
    return s


# (nx, nv, set-up, field amplitude, band rows, columns per CTA)
SHAPES = [
    (64, 256, "two_stream", 0.02, 8, 256),
    (128, 512, "two_stream", 0.3, 16, 256),
    (128, 512, "two_stream", 2.0, 8, 256),     # shifts beyond the 4-cell halo
    (96, 512, "bump_on_tail", 0.05, 16, 256),  # 6 bands x 2 chunks over the CTAs: runs cross chunks
    (2048, 512, "two_stream", 0.05, 16, 256),  # x shifts of many cells: windows far from the band
    (64, 512, "two_stream", 0.5, 4, 256),      # a window of four slabs of 4 rows
    (128, 512, "two_stream", 2.0, 8, 128),     # one-warp CTAs over 128 columns
    (96, 512, "bump_on_tail", 0.05, 4, 128),
    (2048, 256, "two_stream", 0.05, 4, 128),
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


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: f"{s[0]}x{s[1]}_{s[2]}_H{s[3]}_R{s[4]}_C{s[5]}")
def test_strip_forward_and_adjoint_match_oracle(shape, record_error):
    nx, nv, kind, amp, rows, cols = shape
    m, f_eq, f_iv, H = _setup(nx, nv, kind, amp)
    T, dt = 6, 0.05
    s = _solver(m, dt, f_eq, rows, cols, checkpoint_every=3)
    out = s.run_forward(f_iv, H, T * dt)
    g = O.grid_from(m)
    ref = O.delta_forward(g, dt, f_eq, f_iv, H, T)
    worst = 0.0
    for arr, r, name in zip(out, ref, FIELDS):
        err = O.rel_err(arr, r)
        worst = max(worst, err)
        assert err < 1e-5, f"{name}: {err:.2e}"
    record_error(f"strip {nx}x{nv} {kind} H{amp} R{rows} C{cols} fwd", worst, 1e-5)
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
    record_error(f"strip {nx}x{nv} {kind} H{amp} R{rows} C{cols} adj", e, 5e-5)
    assert e < 5e-5, f"adjoint {e:.2e}"


def test_strip_checkpoint_recompute_is_bitwise_neutral():
    """The adjoint recomputes checkpoint segments with the forward's strip kernel, so the gradient
    does not depend on the checkpoint interval by a single bit."""
    m, f_eq, f_iv, H = _setup(128, 512, "two_stream", 0.3)
    T, dt = 9, 0.05
    w = O.trapezoid_time_weights(T, dt)
    for cols in (256, 128):
        outs = []
        for every in (1, 2, 4, 0):
            s = _solver(m, dt, f_eq, 8, cols, checkpoint_every=every or None)
            outs.append(s._run_backward(f_iv, H, T * dt, None, None, None, None, w))
        for gf, gH in outs[1:]:
            assert np.array_equal(gf, outs[0][0]) and np.array_equal(gH, outs[0][1])


def test_strip_agrees_with_persistent_and_is_deterministic():
    m, f_eq, f_iv, H = _setup(128, 512, "two_stream", 0.3)
    T, dt = 8, 0.05
    s = _solver(m, dt, f_eq, 16)
    a = s.run_forward(f_iv, H, T * dt)
    b = s.run_forward(f_iv, H, T * dt)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    p = WarpVlasovPoissonSolver(m, dt, f_eq)
    p.plan.set_config(cluster_size=0, persist_rows=8, strip_rows=0)
    c = p.run_forward(f_iv, H, T * dt)
    for x, y, name in zip(a, c, FIELDS):
        assert O.rel_err(x, y) < 2e-6, name


def test_strip_gradient_through_autograd_matches_oracle():
    m, f_eq, f_iv, H = _setup(64, 512, "two_stream", 0.1)
    T, dt = 7, 0.05
    s = _solver(m, dt, f_eq, 8, checkpoint_every=3)
    Ht = torch.tensor(H, dtype=torch.float32, device="cuda", requires_grad=True)
    fiv = torch.tensor(f_iv, dtype=torch.float64, device="cuda")
    _, _, _, ee = s.run_forward_torch(fiv, Ht, T * dt)
    J = ee.sum() * dt
    J.backward()
    w = np.full(T, dt)
    _, rH = O.delta_backward(O.grid_from(m), dt, f_eq, f_iv, H, T, np.zeros((m.nx, m.nv)), None,
                             np.zeros((T, m.nx)), w)
    assert O.rel_err(Ht.grad.cpu().numpy(), rH) < 5e-5
