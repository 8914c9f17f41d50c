"""CPU restatement of the x-slab calls (vp_slab_* of the C ABI), for testing the slab host loop.

TEST INFRASTRUCTURE ONLY. Nothing in the product package imports this file. The multi-rank
tests inject :class:`OracleSlabOps` into ``warp_vp_solver_b200.slab.SlabSolver`` so that the
product's host loop (ghost-row exchanges, row-sum gathers, checkpoint replay) runs on gloo ranks
without a GPU, and its results are compared with the whole-grid float64 delta oracle
(``vp_oracle.delta_forward`` / ``delta_backward``, the index-space form of
warp_vp_solver/solver.py:418-612 and 742-1105).

Each call applies the delta oracle's per-stage helpers to a slab's array as if it were a periodic
grid of ext_rows rows, exactly as the CUDA calls launch the per-column kernels: the owned rows
read only owned and ghost rows, the other rows' results are discarded. Arrays are float64 CPU
torch tensors; the field record is a small object holding float64 arrays.
"""

from __future__ import annotations

import numpy as np
import torch

import vp_oracle as O


class _Field:
    __slots__ = ("E", "m", "t")

    def __init__(self):
        self.E = self.m = self.t = None


class OracleSlabOps:
    """The slab calls on CPU in float64 (same arguments and semantics as slab.CudaSlabOps)."""

    def __init__(self, grid: O.Grid, dt: float, f_eq_row, row0: int, n_rows: int, pad: int = 1):
        self.g = grid
        self.dt = float(dt)
        self.feq = np.asarray(f_eq_row, np.float64).reshape(-1)
        if self.feq.shape != (grid.nv,):
            raise ValueError("x slabs need an x-invariant f_eq (one row of nv values)")
        self.mx, self.tx = O.x_shift_table(grid, dt)
        lo, hi = int(self.mx.min()), int(self.mx.max())
        self.ghost = max(-2 * lo, 2 * hi + 2, 1)
        if self.ghost > n_rows:
            raise ValueError(f"a slab of {n_rows} rows is thinner than its {self.ghost} ghost rows")
        self.row0, self.n_rows = int(row0), int(n_rows)
        self.ext_rows = n_rows + 2 * self.ghost + int(pad)
        self.rows = (row0 - self.ghost + np.arange(self.ext_rows)) % grid.nx   # grid row of each array row
        self.wv = O._trap_w(grid.nv)
        self.wx = O._trap_w(grid.nx)
        self.mult = O.fft_inv_multiplier(grid.nx, grid.period_x)
        self.device = torch.device("cpu")
        self.field_bytes = 0

    # ---------------------------------------------------------------- helpers
    def new_field(self):
        return _Field()

    def _own(self, a):
        return a[self.ghost:self.ghost + self.n_rows]

    @staticmethod
    def _np(t):
        return t.detach().numpy()

    @staticmethod
    def _put(t, a):
        t.copy_(torch.from_numpy(np.ascontiguousarray(a)).to(t.dtype))

    def _feq_ext(self):
        return np.broadcast_to(self.feq, (self.ext_rows, self.g.nv))

    def _slope(self, h, m, t):
        """f(j + m + 1) - f(j + m) of h + f_eq on every row (the v step's slope)."""
        F = h + self.feq[None, :]
        nv = self.g.nv
        j = np.arange(nv)[None, :]
        i = np.arange(h.shape[0])[:, None]
        return F[i, (j + m[:, None] + 1) % nv] - F[i, (j + m[:, None]) % nv]

    # ---------------------------------------------------------------- forward
    def forward_start(self, f_iv_ext, h_ext, row_sums):
        delta = self._np(f_iv_ext) - self.feq[None, :]
        h = O._x_apply(delta, self.mx, self.tx)
        self._put(h_ext, h)
        self._put(row_sums, self._own(h) @ self.wv)

    def field(self, sums_all, H, field, E_hist_row=None, ee=None):
        rho = -self.g.dv * self._np(sums_all)
        E = O.solve_poisson(rho, self.g.period_x, self.mult)
        Et = E + self._np(H)
        field.E = E
        field.m, field.t = O.v_shift(Et, self.g, self.dt)
        if E_hist_row is not None:
            self._put(E_hist_row, Et)
        if ee is not None:
            self._put(ee, np.array([0.5 * self.g.dx * float(self.wx @ (E * E))]))

    def forward_step(self, h_ext, field, h_out_ext, row_sums, f_rows=None, f_final_rows=None):
        m, t = field.m[self.rows], field.t[self.rows]
        h = self._np(h_ext)
        o = O._v_apply(h, m, t) + O._v_corr(self._feq_ext(), m, t)
        d = O._x_apply(o, self.mx, self.tx)
        if f_rows is not None:
            self._put(f_rows, self._own(d) + self.feq[None, :])
        if f_final_rows is not None:
            self._put(f_final_rows, self._own(d) + self.feq[None, :])
        if h_out_ext is not None:
            hn = O._x_apply(d, self.mx, self.tx)
            self._put(h_out_ext, hn)
            if row_sums is not None:
                self._put(row_sums, self._own(hn) @ self.wv)

    # ---------------------------------------------------------------- adjoint
    def _slope_sums(self, h_prev_ext, field_prev, w):
        m, t = field_prev.m[self.rows], field_prev.t[self.rows]
        sl = self._slope(self._np(h_prev_ext), m, t)
        return self._own(sl * w).sum(axis=1)

    def backward_start(self, g_f_ext, h_prev_ext, field_prev, w_out_ext, slope_sums):
        if g_f_ext is None:
            w = np.zeros((self.ext_rows, self.g.nv))
            self._put(w_out_ext, w)
            self._put(slope_sums, np.zeros(self.n_rows))
            return
        w = O._x_adjoint(self._np(g_f_ext), self.mx, self.tx)
        self._put(w_out_ext, w)
        self._put(slope_sums, self._slope_sums(h_prev_ext, field_prev, w))

    def backward_field(self, slope_all, field_prev, gE_row, gee, g_H, grho):
        g = self.g
        gEt = (-self.dt / g.dv) * self._np(slope_all)
        if gE_row is not None:
            gEt = gEt + self._np(gE_row)
        self._put(g_H, self._np(g_H) + gEt)
        gE = gEt + (0.0 if gee is None else float(self._np(gee)[0])) * g.dx * self.wx * field_prev.E
        self._put(grho, O.solve_poisson_adjoint(gE, g.period_x, self.mult))

    def _gh(self, w_ext, grho, field_n):
        m, t = field_n.m[self.rows], field_n.t[self.rows]
        gh = O._v_adjoint(self._np(w_ext), m, t)
        return gh + (-self.g.dv) * self.wv[None, :] * self._np(grho)[self.rows][:, None]

    def backward_step(self, w_ext, g_f_ext, grho, field_n, field_prev, h_prev_ext, w_out_ext, slope_sums):
        c = O._x_adjoint(self._gh(w_ext, grho, field_n), self.mx, self.tx)
        if g_f_ext is not None:
            c = c + self._np(g_f_ext)
        w = O._x_adjoint(c, self.mx, self.tx)
        self._put(w_out_ext, w)
        self._put(slope_sums, self._slope_sums(h_prev_ext, field_prev, w))

    def backward_finish(self, w_ext, grho, field0, g_f_iv_rows):
        g = O._x_adjoint(self._gh(w_ext, grho, field0), self.mx, self.tx)
        self._put(g_f_iv_rows, self._own(g))
