"""CPU oracle for the Strang-split 1D-1V Vlasov-Poisson step and its discrete adjoint.

TEST INFRASTRUCTURE ONLY. Nothing in the product package imports this file.
Only the tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg use it, always as the checker or as the timed CPU baseline, never as the
path that produces results.

Two flavours, both in float64 NumPy:

(i) ``literal``: a restatement of the reference (Forgotten/warp_vp_solver)
    in the reference's own operation order. Each function cites the file:line
    it follows. The scatter adjoints use ``np.add.at`` in the reference's
    row-major thread order. The trapezoid sums are sequential, as in the
    reference's one-thread-per-row loops. No fused multiply-add is used. This
    flavour is pinned bit-for-bit to golden vectors recorded from the
    reference's own kernels (``tests/golden/make_golden.py``).

(ii) ``delta``: the same scheme re-associated the way the CUDA kernels
    evaluate it. The state is delta = f - f_eq. The semi-Lagrangian feet are
    in index space: an x half-step shifts column j by s_j = 0.5*v_j*dt/dx
    cells, and the v step shifts row i by s_i = (E_i + H_i)*dt/dv cells. Each
    is split once into an integer cell offset m = floor(-s) and a weight
    t = -s - m. In exact arithmetic this equals (i). In float64 the two agree
    to ~1e-13. This is the FP64 oracle "of the same scheme" against which both
    the float32 build and the reference are measured.
"""

from __future__ import annotations

import dataclasses

import numpy as np

# ---------------------------------------------------------------------------
# Grid description (mirrors warp_vp_solver/mesh.py:10-56)
# ---------------------------------------------------------------------------


@dataclasses.dataclass
class Grid:
    xs: np.ndarray
    vs: np.ndarray
    dx: float
    dv: float
    period_x: float      # length_x
    period_v: float      # half width length_v (the v period is 2*period_v)
    nx: int
    nv: int


def make_grid(length_x: float, length_v: float, nx: int, nv: int) -> Grid:
    """Same construction as ``make_mesh`` (warp_vp_solver/mesh.py:26-56)."""
    xs = np.linspace(0.0, length_x, nx, endpoint=False, dtype=np.float64)
    vs = np.linspace(-length_v, length_v, nv, endpoint=False, dtype=np.float64)
    return Grid(xs=xs, vs=vs, dx=float(xs[1] - xs[0]), dv=float(vs[1] - vs[0]),
                period_x=float(length_x), period_v=float(length_v), nx=int(nx), nv=int(nv))


def grid_from(mesh) -> Grid:
    """Accept any object with the Mesh attributes (the package's Mesh, a Grid, ...)."""
    return Grid(xs=np.asarray(mesh.xs, np.float64), vs=np.asarray(mesh.vs, np.float64),
                dx=float(mesh.dx), dv=float(mesh.dv), period_x=float(mesh.period_x),
                period_v=float(mesh.period_v), nx=int(mesh.nx), nv=int(mesh.nv))


# ---------------------------------------------------------------------------
# (i) literal restatement
# ---------------------------------------------------------------------------


def periodic_indices(x_query, x0, h, n, period):
    """warp_vp_solver/kernels.py:47-69 (vectorised, same operation order)."""
    x_rel = x_query - x0
    x_wrapped = x_rel - np.floor(x_rel / period) * period
    idx_f = x_wrapped / h
    i0 = np.floor(idx_f).astype(np.int64) % n
    i0 = np.where(i0 < 0, i0 + n, i0)
    i1 = (i0 + 1) % n
    t = idx_f - np.floor(idx_f)
    return i0, i1, t


def semilag_x(f, g: Grid, dt):
    """X_{dt/2}: warp_vp_solver/kernels.py:109-130 with periodic_interp_col (72-85)."""
    x_foot = g.xs[:, None] - 0.5 * g.vs[None, :] * dt
    i0, i1, t = periodic_indices(x_foot, g.xs[0], g.dx, g.nx, g.period_x)
    j = np.broadcast_to(np.arange(g.nv)[None, :], x_foot.shape)
    return (1.0 - t) * f[i0, j] + t * f[i1, j]


def semilag_v(f, E_total, g: Grid, dt):
    """V_dt: warp_vp_solver/kernels.py:133-153 (period 2*length_v, solver.py:241)."""
    v_foot = g.vs[None, :] - E_total[:, None] * dt
    i0, i1, t = periodic_indices(v_foot, g.vs[0], g.dv, g.nv, 2.0 * g.period_v)
    i = np.broadcast_to(np.arange(g.nx)[:, None], v_foot.shape)
    return (1.0 - t) * f[i, i0] + t * f[i, i1]


def semilag_v_fused(f, E, H, g: Grid, dt):
    """warp_vp_solver/kernels.py:367-393: E_total = E + H formed per row."""
    return semilag_v(f, E + H, g, dt)


def compute_rho(f_eq, f, dv):
    """warp_vp_solver/kernels.py:156-172: sequential trapezoid of (f_eq - f) along v."""
    nv = f.shape[1]
    d = f_eq - f
    acc = 0.5 * d[:, 0]
    for k in range(1, nv - 1):
        acc = acc + d[:, k]
    acc = acc + 0.5 * d[:, nv - 1]
    return acc * dv


def compute_ee(E, dx):
    """warp_vp_solver/kernels.py:175-197: sequential 0.5*trapz(E^2)*dx."""
    nx = E.shape[0]
    acc = 0.5 * E[0] * E[0]
    for k in range(1, nx - 1):
        acc = acc + E[k] * E[k]
    acc = acc + 0.5 * E[nx - 1] * E[nx - 1]
    return 0.5 * acc * dx


def semilag_x_adjoint(g_out, g: Grid, dt):
    """warp_vp_solver/kernels.py:215-241: scatter with the lerp weights."""
    x_foot = g.xs[:, None] - 0.5 * g.vs[None, :] * dt
    i0, i1, t = periodic_indices(x_foot, g.xs[0], g.dx, g.nx, g.period_x)
    j = np.broadcast_to(np.arange(g.nv)[None, :], x_foot.shape)
    rows = np.stack([i0, i1], axis=-1).reshape(-1)
    cols = np.stack([j, j], axis=-1).reshape(-1)
    vals = np.stack([(1.0 - t) * g_out, t * g_out], axis=-1).reshape(-1)
    g_in = np.zeros_like(g_out)
    np.add.at(g_in, (rows, cols), vals)
    return g_in


def semilag_v_adjoint(g_out, f_in, E_total, g: Grid, dt):
    """warp_vp_solver/kernels.py:244-273 (and the fused form 396-429).

    Returns ``(g_in, g_E_total)``.
    """
    v_foot = g.vs[None, :] - E_total[:, None] * dt
    i0, i1, t = periodic_indices(v_foot, g.vs[0], g.dv, g.nv, 2.0 * g.period_v)
    i = np.broadcast_to(np.arange(g.nx)[:, None], v_foot.shape)
    rows = np.stack([i, i], axis=-1).reshape(-1)
    cols = np.stack([i0, i1], axis=-1).reshape(-1)
    vals = np.stack([(1.0 - t) * g_out, t * g_out], axis=-1).reshape(-1)
    g_in = np.zeros_like(g_out)
    np.add.at(g_in, (rows, cols), vals)
    df_dvfoot = (f_in[i, i1] - f_in[i, i0]) / g.dv
    g_E = np.zeros(g.nx)
    np.add.at(g_E, i.reshape(-1), (-dt * df_dvfoot * g_out).reshape(-1))
    return g_in, g_E


def compute_rho_adjoint(g_rho, nv, dv, g_f=None):
    """warp_vp_solver/kernels.py:276-299: g_f[i,j] += w_j g_rho[i]."""
    w = np.full(nv, -dv)
    w[0] = -0.5 * dv
    w[nv - 1] = -0.5 * dv
    base = np.zeros((g_rho.shape[0], nv)) if g_f is None else g_f
    return base + w[None, :] * g_rho[:, None]


def compute_ee_adjoint(g_ee, E, dx, g_E=None):
    """warp_vp_solver/kernels.py:302-322: g_E[k] += w_k E[k] g_ee."""
    nx = E.shape[0]
    w = np.full(nx, dx)
    w[0] = 0.5 * dx
    w[nx - 1] = 0.5 * dx
    base = np.zeros(nx) if g_E is None else g_E
    return base + w * E * g_ee


def fft_inv_multiplier(nx, period_x):
    """warp_vp_solver/poisson.py:34-45."""
    freqs = np.fft.fftfreq(nx, d=period_x / nx)
    mult = np.zeros(nx, dtype=np.complex128)
    nz = freqs != 0.0
    mult[nz] = -1.0 / (1j * 2.0 * np.pi * freqs[nz])
    return mult


def solve_poisson(rho, period_x, mult=None):
    """warp_vp_solver/poisson.py:48-69."""
    if mult is None:
        mult = fft_inv_multiplier(rho.shape[0], period_x)
    return np.real(np.fft.ifft(mult * np.fft.fft(rho)))


def solve_poisson_adjoint(g_E, period_x, mult=None):
    """warp_vp_solver/poisson.py:72-99."""
    if mult is None:
        mult = fft_inv_multiplier(g_E.shape[0], period_x)
    return np.real(np.fft.ifft(np.conj(mult) * np.fft.fft(g_E)))


def num_steps(t_final, dt):
    """warp_vp_solver/solver.py:212-213."""
    return int(t_final / dt)


def run_forward(g: Grid, dt, f_eq, f_iv, H, t_final):
    """Legacy forward loop, warp_vp_solver/solver.py:470-524.

    Returns ``(f_final, f_hist, E_hist, ee_hist)``; ``E_hist`` holds E + H and
    ``ee_hist`` the energy of E alone.
    """
    T = num_steps(t_final, dt)
    f_eq = np.asarray(f_eq, np.float64)
    H = np.asarray(H, np.float64)
    mult = fft_inv_multiplier(g.nx, g.period_x)
    f = np.array(f_iv, dtype=np.float64, copy=True)
    f_hist = np.empty((T, g.nx, g.nv))
    E_hist = np.empty((T, g.nx))
    ee_hist = np.empty(T)
    for t in range(T):
        f_half = semilag_x(f, g, dt)
        rho = compute_rho(f_eq, f_half, g.dv)
        E = solve_poisson(rho, g.period_x, mult)
        ee = compute_ee(E, g.dx)
        E_total = E + H
        f_one = semilag_v(f_half, E_total, g, dt)
        f = semilag_x(f_one, g, dt)
        f_hist[t] = f
        E_hist[t] = E_total
        ee_hist[t] = ee
    f_final = f_hist[-1].copy() if T > 0 else np.array(f_iv, dtype=np.float64, copy=True)
    return f_final, f_hist, E_hist, ee_hist


def run_backward(g: Grid, dt, f_eq, f_iv, H, t_final, f_hist,
                 g_f_final, g_f_hist, g_E_hist, g_ee_hist):
    """Legacy discrete adjoint, warp_vp_solver/solver.py:778-932.

    Returns ``(g_f_iv, g_H)``.
    """
    T = num_steps(t_final, dt)
    f_eq = np.asarray(f_eq, np.float64)
    f_iv = np.asarray(f_iv, np.float64)
    H = np.asarray(H, np.float64)
    mult = fft_inv_multiplier(g.nx, g.period_x)
    g_f = np.array(g_f_final, dtype=np.float64, copy=True)
    g_H = np.zeros(g.nx)
    for t in range(T - 1, -1, -1):
        f_step_in = f_iv if t == 0 else f_hist[t - 1]
        g_f = g_f + np.asarray(g_f_hist[t], np.float64)
        f_half = semilag_x(f_step_in, g, dt)
        rho = compute_rho(f_eq, f_half, g.dv)
        E = solve_poisson(rho, g.period_x, mult)
        E_total = E + H
        g_f_one = semilag_x_adjoint(g_f, g, dt)
        g_f_half_v, g_E_total_from_v = semilag_v_adjoint(g_f_one, f_half, E_total, g, dt)
        g_E_total = g_E_total_from_v + np.asarray(g_E_hist[t], np.float64)
        g_H = g_H + g_E_total
        g_E = compute_ee_adjoint(float(g_ee_hist[t]), E, g.dx, g_E_total.copy())
        g_rho = solve_poisson_adjoint(g_E, g.period_x, mult)
        g_f_half = g_f_half_v + compute_rho_adjoint(g_rho, g.nv, g.dv)
        g_f = semilag_x_adjoint(g_f_half, g, dt)
    return g_f, g_H


# ---------------------------------------------------------------------------
# (ii) index-space delta-f flavour (the scheme the CUDA kernels evaluate)
# ---------------------------------------------------------------------------


def run_forward_aggressive(g: Grid, dt, f_eq, f_iv, H, t_final):
    """Merged-Strang forward, warp_vp_solver/solver.py:618-736: the trailing X(dt/2) of a step and
    the leading X(dt/2) of the next are one X(dt) (``semilag_x_full_kernel``, kernels.py:535-556;
    a full step is the half-step form with 2*dt). ``f_hist[t]`` is the state after the merged
    X(dt) (``f_final`` for the last step). Returns ``(f_final, f_hist, E_hist, ee_hist)``."""
    T = num_steps(t_final, dt)
    f_eq = np.asarray(f_eq, np.float64)
    H = np.asarray(H, np.float64)
    f_hist = np.empty((T, g.nx, g.nv))
    E_hist = np.empty((T, g.nx))
    ee_hist = np.empty(T)
    f_half = semilag_x(np.asarray(f_iv, np.float64), g, dt)
    rho = compute_rho(f_eq, f_half, g.dv)
    f_final = f_half
    for t in range(T):
        E = solve_poisson(rho, g.period_x)
        ee = compute_ee(E, g.dx)
        post_v = semilag_v(f_half, E + H, g, dt)
        if t < T - 1:
            f_half = semilag_x(post_v, g, 2.0 * dt)
            rho = compute_rho(f_eq, f_half, g.dv)
            f_hist[t] = f_half
        else:
            f_final = semilag_x(post_v, g, dt)
            f_hist[t] = f_final
        E_hist[t] = E + H
        ee_hist[t] = ee
    return f_final, f_hist, E_hist, ee_hist


def run_backward_aggressive(g: Grid, dt, f_eq, f_iv, H, t_final, f_hist,
                            g_f_final, g_f_hist, g_E_hist, g_ee_hist):
    """Discrete adjoint of :func:`run_forward_aggressive`, warp_vp_solver/solver.py:1111-1338:
    X(dt/2)^T for the last step, X(dt)^T for the merged inner steps, V^T, the E_total, ee,
    Poisson and rho transposes, and X(dt/2)^T of the leading half step. Returns
    ``(g_f_iv, g_H)``."""
    T = num_steps(t_final, dt)
    f_eq = np.asarray(f_eq, np.float64)
    f_iv = np.asarray(f_iv, np.float64)
    H = np.asarray(H, np.float64)
    g_f = np.array(g_f_final, dtype=np.float64, copy=True) + np.asarray(g_f_hist[T - 1], np.float64)
    g_H = np.zeros(g.nx)
    g_f_half = None
    for t in range(T - 1, -1, -1):
        f_half = semilag_x(f_iv, g, dt) if t == 0 else np.asarray(f_hist[t - 1], np.float64)
        rho = compute_rho(f_eq, f_half, g.dv)
        E = solve_poisson(rho, g.period_x)
        g_in = semilag_x_adjoint(g_f, g, dt if t == T - 1 else 2.0 * dt)
        g_f_half, g_E_total = semilag_v_adjoint(g_in, f_half, E + H, g, dt)
        g_E_total = g_E_total + np.asarray(g_E_hist[t], np.float64)
        g_H = g_H + g_E_total
        g_E_back = g_E_total + compute_ee_adjoint(float(g_ee_hist[t]), E, g.dx)
        g_rho = solve_poisson_adjoint(g_E_back, g.period_x)
        g_f_half = g_f_half + compute_rho_adjoint(g_rho, g.nv, g.dv)
        if t > 0:
            g_f = g_f_half + np.asarray(g_f_hist[t - 1], np.float64)
    return semilag_x_adjoint(g_f_half, g, dt), g_H


def x_shift_table(g: Grid, dt):
    """Per-column x half-step: integer offset m_j and weight t_j (float64)."""
    s = 0.5 * g.vs * dt / g.dx
    m = np.floor(-s)
    t = -s - m
    return m.astype(np.int64), t


def v_shift(E_total, g: Grid, dt):
    """Per-row v step: integer offset m_i and weight t_i (float64)."""
    s = E_total * (dt / g.dv)
    m = np.floor(-s)
    t = -s - m
    return m.astype(np.int64), t


def _x_apply(a, m, t):
    nx = a.shape[0]
    i = np.arange(nx)[:, None]
    j = np.arange(a.shape[1])[None, :]
    return (1.0 - t)[None, :] * a[(i + m[None, :]) % nx, j] + t[None, :] * a[(i + m[None, :] + 1) % nx, j]


def _x_corr(f_eq, m, t):
    """X(f_eq) - f_eq in difference form (zero when f_eq is x-invariant)."""
    nx = f_eq.shape[0]
    i = np.arange(nx)[:, None]
    j = np.arange(f_eq.shape[1])[None, :]
    a0 = f_eq[(i + m[None, :]) % nx, j] - f_eq
    a1 = f_eq[(i + m[None, :] + 1) % nx, j] - f_eq
    return (1.0 - t)[None, :] * a0 + t[None, :] * a1


def _v_apply(a, m, t):
    nv = a.shape[1]
    j = np.arange(nv)[None, :]
    i = np.arange(a.shape[0])[:, None]
    return (1.0 - t)[:, None] * a[i, (j + m[:, None]) % nv] + t[:, None] * a[i, (j + m[:, None] + 1) % nv]


def _v_corr(f_eq, m, t):
    nv = f_eq.shape[1]
    j = np.arange(nv)[None, :]
    i = np.arange(f_eq.shape[0])[:, None]
    a0 = f_eq[i, (j + m[:, None]) % nv] - f_eq
    a1 = f_eq[i, (j + m[:, None] + 1) % nv] - f_eq
    return (1.0 - t)[:, None] * a0 + t[:, None] * a1


def _x_adjoint(b, m, t):
    nx = b.shape[0]
    k = np.arange(nx)[:, None]
    j = np.arange(b.shape[1])[None, :]
    return (1.0 - t)[None, :] * b[(k - m[None, :]) % nx, j] + t[None, :] * b[(k - m[None, :] - 1) % nx, j]


def _v_adjoint(b, m, t):
    nv = b.shape[1]
    k = np.arange(nv)[None, :]
    i = np.arange(b.shape[0])[:, None]
    return (1.0 - t)[:, None] * b[i, (k - m[:, None]) % nv] + t[:, None] * b[i, (k - m[:, None] - 1) % nv]


def _trap_w(n):
    w = np.ones(n)
    w[0] = 0.5
    w[-1] = 0.5
    return w


def delta_forward(g: Grid, dt, f_eq, f_iv, H, n_steps, *, keep_half=False):
    """Index-space delta-f forward. Same outputs as :func:`run_forward`.

    With ``keep_half`` also returns the list of delta_half states h_n and the
    raw self-consistent fields E_n (the backward's inputs).
    """
    f_eq = np.asarray(f_eq, np.float64)
    H = np.asarray(H, np.float64)
    mx, tx = x_shift_table(g, dt)
    xc = _x_corr(f_eq, mx, tx)
    wv = _trap_w(g.nv)
    wx = _trap_w(g.nx)
    mult = fft_inv_multiplier(g.nx, g.period_x)
    delta = np.asarray(f_iv, np.float64) - f_eq
    f_hist = np.empty((n_steps, g.nx, g.nv))
    E_hist = np.empty((n_steps, g.nx))
    ee_hist = np.empty(n_steps)
    hs, Es = [], []
    for n in range(n_steps):
        h = _x_apply(delta, mx, tx) + xc
        rho = -g.dv * (h @ wv)
        E = solve_poisson(rho, g.period_x, mult)
        ee = 0.5 * g.dx * float(wx @ (E * E))
        Et = E + H
        mv, tv = v_shift(Et, g, dt)
        o = _v_apply(h, mv, tv) + _v_corr(f_eq, mv, tv)
        delta = _x_apply(o, mx, tx) + xc
        f_hist[n] = delta + f_eq
        E_hist[n] = Et
        ee_hist[n] = ee
        if keep_half:
            hs.append(h)
            Es.append(E)
    f_final = delta + f_eq
    if keep_half:
        return f_final, f_hist, E_hist, ee_hist, hs, Es
    return f_final, f_hist, E_hist, ee_hist


def delta_backward(g: Grid, dt, f_eq, f_iv, H, n_steps,
                   g_f_final, g_f_hist, g_E_hist, g_ee_hist):
    """Index-space discrete adjoint of :func:`delta_forward` (no recompute: keeps every h_n)."""
    f_eq = np.asarray(f_eq, np.float64)
    H = np.asarray(H, np.float64)
    _, _, _, _, hs, Es = delta_forward(g, dt, f_eq, f_iv, H, n_steps, keep_half=True)
    mx, tx = x_shift_table(g, dt)
    wv = _trap_w(g.nv)
    wx = _trap_w(g.nx)
    mult = fft_inv_multiplier(g.nx, g.period_x)
    nv = g.nv
    c = np.array(g_f_final, dtype=np.float64, copy=True)
    g_H = np.zeros(g.nx)
    for n in range(n_steps - 1, -1, -1):
        if g_f_hist is not None:
            c = c + g_f_hist[n]
        w = _x_adjoint(c, mx, tx)
        E = Es[n]
        Et = E + H
        mv, tv = v_shift(Et, g, dt)
        gh = _v_adjoint(w, mv, tv)
        F = hs[n] + f_eq
        i = np.arange(g.nx)[:, None]
        j = np.arange(nv)[None, :]
        slope = F[i, (j + mv[:, None] + 1) % nv] - F[i, (j + mv[:, None]) % nv]
        gEt = np.sum((-dt / g.dv) * slope * w, axis=1)
        if g_E_hist is not None:
            gEt = gEt + g_E_hist[n]
        g_H = g_H + gEt
        gE = gEt + (0.0 if g_ee_hist is None else g_ee_hist[n]) * g.dx * wx * E
        g_rho = solve_poisson_adjoint(gE, g.period_x, mult)
        gh = gh + (-g.dv) * wv[None, :] * g_rho[:, None]
        c = _x_adjoint(gh, mx, tx)
    return c, g_H


# ---------------------------------------------------------------------------
# Problem set-ups and costs used by the parity cases
# ---------------------------------------------------------------------------


def external_electric_field(coeffs, xs, k0):
    """warp_vp_solver/utils.py:37-48 in NumPy: sum_k a_k cos(k0 k x) + b_k sin(k0 k x)."""
    coeffs = np.asarray(coeffs, np.float64)
    n = coeffs.shape[1]
    k = np.arange(1, n + 1)
    return coeffs[0] @ np.cos(k0 * k[:, None] * xs) + coeffs[1] @ np.sin(k0 * k[:, None] * xs)


def trapezoid_time_weights(n_steps, dt):
    """dJ/dee for J = trapezoid(ee, dx=dt) (warp_vp_solver/utils.py:111-116)."""
    if n_steps < 2:
        return np.zeros(n_steps)
    w = np.full(n_steps, float(dt))
    w[0] *= 0.5
    w[-1] *= 0.5
    return w


def rel_err(a, b):
    """max|a-b| / max|b| (infinity-norm relative error)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / den) if den > 0 else float(np.max(np.abs(a - b)))
