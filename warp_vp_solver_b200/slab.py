"""x-slab decomposition: one grid split into slabs of consecutive x rows, one slab per device.

The reference solves a whole grid on one Warp device (warp_vp_solver/solver.py:170-203). For a
grid whose state does not fit one GPU, the rows split into slabs. A Strang step reads, for an
output row r, rows r + 2m .. r + 2m + 2 of the step's input (m: the x half-step offsets of the
columns), so each slab keeps ``ghost`` copied rows of each neighbour; the rho of the next step is
a sum over v inside each row, so the slabs' row sums are gathered (one all-gather of nx values)
and every rank solves the same Poisson problem on them. Per step, then: one ghost-row exchange
with the two neighbours and one all-gather of nx reals, forward and adjoint alike. The adjoint
recomputes each rank's own slab from checkpoints (every K = ceil(sqrt(T)) steps), replaying the
same exchanges, so every rank takes the same collective steps in the same order.

Pieces:
  * :func:`slab_bounds` - the rows of each slab;
  * :class:`LocalRing` - every slab of the grid in this process (one device; the ranks' steps run
    one after the other and the exchanges are copies);
  * :class:`DistRing` - one slab per rank of a ``torch.distributed`` group (NCCL over NVLink on
    GPUs, gloo on CPU): ghost rows by point-to-point sends to the two neighbours, row sums by one
    ``all_gather``;
  * :class:`CudaSlabOps` - the slab calls of the C ABI (``vp_slab_*``) on one device;
  * :class:`SlabSolver` - the forward loop and the checkpointed discrete adjoint over a ring.
The per-slab operations are injectable (``ops_factory``), so the host loop and the ring can be
tested on CPU ranks with a CPU restatement of the slab calls.
"""

from __future__ import annotations

import ctypes
import math
from typing import Callable

import numpy as np
import torch
import torch.distributed as dist

from . import _capi
from .plan import Plan, as_torch_dtype


def slab_bounds(nx: int, n_slabs: int) -> list[tuple[int, int]]:
    """(first row, rows) of each slab: consecutive, sizes differing by at most one."""
    if n_slabs < 1 or n_slabs > nx:
        raise ValueError(f"cannot split {nx} rows into {n_slabs} slabs")
    edges = [(k * nx) // n_slabs for k in range(n_slabs + 1)]
    return [(edges[k], edges[k + 1] - edges[k]) for k in range(n_slabs)]


def _owned(a: torch.Tensor, ghost: int, n_rows: int) -> torch.Tensor:
    return a[ghost:ghost + n_rows]


class LocalRing:
    """Every slab of the grid in this process: exchanges are device copies, the gather a concat."""

    def __init__(self, n_slabs: int):
        self.n_slabs = int(n_slabs)
        self.local = list(range(self.n_slabs))

    def exchange(self, arrays: dict, ghost: int, rows: dict) -> None:
        """Fills the ghost rows of every slab's array from its neighbours' owned rows."""
        n = self.n_slabs
        for s in self.local:
            lo, hi = (s - 1) % n, (s + 1) % n
            a = arrays[s]
            a[0:ghost].copy_(arrays[lo][rows[lo]:rows[lo] + ghost])
            a[ghost + rows[s]:2 * ghost + rows[s]].copy_(arrays[hi][ghost:2 * ghost])

    def gather_rows(self, parts: dict, rows: dict) -> torch.Tensor:
        """The slabs' row arrays in grid-row order (one array of nx values)."""
        return torch.cat([parts[s][:rows[s]] for s in self.local])


class DistRing:
    """One slab per rank of a ``torch.distributed`` process group (slab index = group rank).

    Ghost rows travel by point-to-point operations to the two neighbours (periodic in x): each
    rank sends its top ``ghost`` owned rows up and its bottom ones down, posted in the same order
    on every rank (sends up, sends down, receive from below, receive from above), so NCCL's
    in-order matching and gloo's tags pair them the same way for any number of ranks. Row sums
    travel by one ``all_gather`` (padded to the largest slab)."""

    def __init__(self, group=None):
        if not dist.is_initialized():
            raise RuntimeError("DistRing needs an initialised torch.distributed process group")
        self.group = group
        self.rank = dist.get_rank(group)
        self.n_slabs = dist.get_world_size(group)
        self.local = [self.rank]

    def _peer(self, s: int) -> int:
        return s if self.group is None else dist.get_global_rank(self.group, s)

    def exchange(self, arrays: dict, ghost: int, rows: dict) -> None:
        s = self.rank
        a = arrays[s]
        n = rows[s]
        up_send, down_send = a[n:n + ghost], a[ghost:2 * ghost]
        lo_recv, hi_recv = a[0:ghost], a[ghost + n:2 * ghost + n]
        if self.n_slabs == 1:
            lo_recv.copy_(up_send)
            hi_recv.copy_(down_send)
            return
        up, down = self._peer((s + 1) % self.n_slabs), self._peer((s - 1) % self.n_slabs)
        ops = [dist.P2POp(dist.isend, up_send.contiguous(), up, self.group, tag=1),
               dist.P2POp(dist.isend, down_send.contiguous(), down, self.group, tag=2),
               dist.P2POp(dist.irecv, lo_recv, down, self.group, tag=1),
               dist.P2POp(dist.irecv, hi_recv, up, self.group, tag=2)]
        for req in dist.batch_isend_irecv(ops):
            req.wait()

    def gather_rows(self, parts: dict, rows: dict) -> torch.Tensor:
        s = self.rank
        width = max(rows.values()) if len(rows) == self.n_slabs else None
        if width is None:
            raise ValueError("DistRing.gather_rows needs every slab's row count")
        mine = parts[s]
        buf = torch.zeros(width, dtype=mine.dtype, device=mine.device)
        buf[:rows[s]].copy_(mine[:rows[s]])
        out = [torch.empty_like(buf) for _ in range(self.n_slabs)]
        dist.all_gather(out, buf, group=self.group)
        return torch.cat([out[k][:rows[k]] for k in range(self.n_slabs)])


class CudaSlabOps:
    """The ``vp_slab_*`` calls of the C ABI for one slab of a plan (device tensors)."""

    def __init__(self, plan: Plan, row0: int, n_rows: int):
        self.plan = plan
        self.lib = plan.lib
        self.device = plan.device
        self.dtype = plan.dtype
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _capi.check(self.lib.vp_slab_create(plan.handle, int(row0), int(n_rows), ctypes.byref(h)))
        self._h = h
        g, e, fb = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_size_t()
        _capi.check(self.lib.vp_slab_geometry(h, ctypes.byref(g), ctypes.byref(e), ctypes.byref(fb)))
        self.ghost, self.ext_rows, self.field_bytes = int(g.value), int(e.value), int(fb.value)

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.vp_slab_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------- buffers
    def new_field(self) -> torch.Tensor:
        # torch's caching allocator returns 512-byte aligned blocks; the call checks 256
        return torch.empty(self.field_bytes, dtype=torch.uint8, device=self.device)

    @staticmethod
    def _p(t):
        return None if t is None else t.data_ptr()

    def _s(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    # ---------------------------------------------------------------- calls
    def forward_start(self, f_iv_ext, h_ext, row_sums):
        _capi.check(self.lib.vp_slab_forward_start(self._h, f_iv_ext.data_ptr(), h_ext.data_ptr(),
                                                   row_sums.data_ptr(), self._s()))

    def field(self, sums_all, H, field, E_hist_row=None, ee=None):
        _capi.check(self.lib.vp_slab_field(self._h, sums_all.data_ptr(), H.data_ptr(), field.data_ptr(),
                                           self._p(E_hist_row), self._p(ee), self._s()))

    def forward_step(self, h_ext, field, h_out_ext, row_sums, f_rows=None, f_final_rows=None):
        p = self._p
        _capi.check(self.lib.vp_slab_forward_step(self._h, h_ext.data_ptr(), field.data_ptr(), p(h_out_ext),
                                                  p(row_sums), p(f_rows), p(f_final_rows), self._s()))

    def backward_start(self, g_f_ext, h_prev_ext, field_prev, w_out_ext, slope_sums):
        _capi.check(self.lib.vp_slab_backward_start(self._h, self._p(g_f_ext), h_prev_ext.data_ptr(),
                                                    field_prev.data_ptr(), w_out_ext.data_ptr(),
                                                    slope_sums.data_ptr(), self._s()))

    def backward_field(self, slope_all, field_prev, gE_row, gee, g_H, grho):
        _capi.check(self.lib.vp_slab_backward_field(self._h, slope_all.data_ptr(), field_prev.data_ptr(),
                                                    self._p(gE_row), self._p(gee), g_H.data_ptr(), grho.data_ptr(),
                                                    self._s()))

    def backward_step(self, w_ext, g_f_ext, grho, field_n, field_prev, h_prev_ext, w_out_ext, slope_sums):
        _capi.check(self.lib.vp_slab_backward_step(self._h, w_ext.data_ptr(), self._p(g_f_ext), grho.data_ptr(),
                                                   field_n.data_ptr(), field_prev.data_ptr(), h_prev_ext.data_ptr(),
                                                   w_out_ext.data_ptr(), slope_sums.data_ptr(), self._s()))

    def backward_finish(self, w_ext, grho, field0, g_f_iv_rows):
        _capi.check(self.lib.vp_slab_backward_finish(self._h, w_ext.data_ptr(), grho.data_ptr(), field0.data_ptr(),
                                                     g_f_iv_rows.data_ptr(), self._s()))


class SlabSolver:
    """Forward loop and checkpointed discrete adjoint of one grid split into x slabs over a ring.

    ``ring`` is a :class:`LocalRing` or a :class:`DistRing`; this process holds the slabs in
    ``ring.local``. Row arguments and results are dicts slab index -> (n_rows, nv) array of that
    slab's owned rows; field quantities (H, E_hist, ee_hist, g_H) are whole-grid arrays that every
    rank holds. ``ops_factory(row0, n_rows)`` builds the per-slab calls (default: the CUDA ones on
    a plan of this grid on ``device``)."""

    def __init__(self, mesh, dt: float, f_eq, ring, *, dtype=torch.float32, device=None,
                 ops_factory: Callable | None = None):
        self.mesh = mesh
        self.nx, self.nv = int(mesh.nx), int(mesh.nv)
        self.dt = float(dt)
        self.ring = ring
        self.dtype = as_torch_dtype(dtype)
        self.bounds = slab_bounds(self.nx, ring.n_slabs)
        self.rows = {s: self.bounds[s][1] for s in range(ring.n_slabs)}
        if ops_factory is None:
            f_eq = np.asarray(f_eq, dtype=np.float64)
            if f_eq.ndim == 2:   # x slabs need an x-invariant f_eq: keep its first row
                if not (f_eq == f_eq[:1]).all():
                    raise ValueError("x slabs need an x-invariant f_eq (every row equal)")
                f_eq = f_eq[0]
            # the plan is built from the row alone: no (nx, nv) host array for a grid too large
            # for one GPU
            self.plan = Plan(mesh, dt, f_eq, dtype=self.dtype, device=device)
            ops_factory = lambda row0, n_rows: CudaSlabOps(self.plan, row0, n_rows)   # noqa: E731
        self.ops = {s: ops_factory(*self.bounds[s]) for s in ring.local}
        first = self.ops[ring.local[0]]
        self.ghost = first.ghost
        self.device = first.device
        self.field_op = first   # the field is solved once per process (every rank gets the same)

    # ---------------------------------------------------------------- helpers
    def num_steps(self, t_final: float) -> int:
        """T = int(t_final / dt) (warp_vp_solver/solver.py:443)."""
        return int(float(t_final) / self.dt)

    def _ext(self, s: int, dtype) -> torch.Tensor:
        return torch.zeros((self.ops[s].ext_rows, self.nv), dtype=dtype, device=self.device)

    def _place(self, rows_in: dict, dtype) -> dict:
        out = {}
        for s in self.ring.local:
            a = self._ext(s, dtype)
            src = torch.as_tensor(rows_in[s]).to(device=self.device, dtype=dtype)
            if tuple(src.shape) != (self.rows[s], self.nv):
                raise ValueError(f"slab {s}: rows of shape {tuple(src.shape)} != ({self.rows[s]}, {self.nv})")
            _owned(a, self.ghost, self.rows[s]).copy_(src)
            out[s] = a
        self.ring.exchange(out, self.ghost, self.rows)
        return out

    def _real(self, a, shape) -> torch.Tensor:
        t = torch.as_tensor(a).to(device=self.device, dtype=self.dtype).contiguous()
        if tuple(t.shape) != tuple(shape):
            raise ValueError(f"expected shape {tuple(shape)}, got {tuple(t.shape)}")
        return t

    def _sums(self) -> dict:
        return {s: torch.empty(self.rows[s], dtype=self.dtype, device=self.device) for s in self.ring.local}

    # ---------------------------------------------------------------- forward
    def _forward(self, f_iv_rows: dict, H: torch.Tensor, T: int, *, record_history: bool, every: int = 0):
        L, G = self.ring.local, self.ghost
        f_iv = self._place(f_iv_rows, torch.float64)
        h = {s: self._ext(s, self.dtype) for s in L}
        h_next = {s: self._ext(s, self.dtype) for s in L}
        sums = self._sums()
        E_hist = torch.empty((T, self.nx), dtype=self.dtype, device=self.device)
        ee_hist = torch.empty(T, dtype=self.dtype, device=self.device)
        fields = [self.field_op.new_field() for _ in range(T if every else 2)]
        f_hist = {s: torch.empty((T, self.rows[s], self.nv), dtype=self.dtype, device=self.device) for s in L} \
            if record_history else None
        f_final = {s: torch.empty((self.rows[s], self.nv), dtype=torch.float64, device=self.device) for s in L}
        ckpt = []
        for s in L:
            self.ops[s].forward_start(f_iv[s], h[s], sums[s])
        del f_iv
        self.field_op.field(self.ring.gather_rows(sums, self.rows), H, fields[0], E_hist[0], ee_hist[0:1])
        for n in range(T):
            last = n == T - 1
            self.ring.exchange(h, G, self.rows)
            if every and n % every == 0:
                ckpt.append({s: h[s].clone() for s in L})
            fld = fields[n] if every else fields[n & 1]
            for s in L:
                self.ops[s].forward_step(h[s], fld, None if last else h_next[s], None if last else sums[s],
                                         f_hist[s][n] if record_history else None, f_final[s] if last else None)
            if not last:
                nxt = fields[n + 1] if every else fields[(n + 1) & 1]
                self.field_op.field(self.ring.gather_rows(sums, self.rows), H, nxt, E_hist[n + 1],
                                    ee_hist[n + 1:n + 2])
                h, h_next = h_next, h
        return f_final, f_hist, E_hist, ee_hist, fields, ckpt

    def run_forward(self, f_iv_rows: dict, H, t_final: float, *, record_history: bool = False):
        """Forward loop (warp_vp_solver/solver.py:418-612) over the slabs.

        Returns (f_final rows, f_history rows or None, E_history (T, nx), ee_history (T,)) with the
        row results as dicts slab index -> array of that slab's owned rows."""
        T = self.num_steps(t_final)
        if T < 1:
            raise ValueError("t_final must give at least one time step")
        H = self._real(H, (self.nx,))
        f_final, f_hist, E_hist, ee_hist, _, _ = self._forward(f_iv_rows, H, T, record_history=record_history)
        return f_final, f_hist, E_hist, ee_hist

    # ---------------------------------------------------------------- adjoint
    def vjp(self, f_iv_rows: dict, H, t_final: float, *, g_E_hist=None, g_ee_hist=None, g_f_final_rows=None,
            checkpoint_every: int | None = None):
        """Discrete adjoint (warp_vp_solver/solver.py:742-1105) of the slab forward loop.

        Cotangents: on E_history (T, nx), on ee_history (T,) and on the final state's owned rows
        (dict of (n_rows, nv)); None means zero. The forward keeps a checkpoint of every slab
        state each ``checkpoint_every`` steps (default ceil(sqrt(T))) and the adjoint replays one
        segment at a time. Returns a dict with ``g_f_iv`` (rows per slab), ``g_H`` (nx),
        ``E_hist`` and ``ee_hist`` of the forward pass."""
        T = self.num_steps(t_final)
        if T < 1:
            raise ValueError("t_final must give at least one time step")
        L, G = self.ring.local, self.ghost
        K = int(checkpoint_every) if checkpoint_every else math.isqrt(T - 1) + 1   # ceil(sqrt(T))
        H = self._real(H, (self.nx,))
        gEh = None if g_E_hist is None else self._real(g_E_hist, (T, self.nx))
        gee = None if g_ee_hist is None else self._real(g_ee_hist, (T,))
        _, _, E_hist, ee_hist, fields, ckpt = self._forward(f_iv_rows, H, T, record_history=False, every=K)

        seg_cache: dict = {"index": -1, "states": {}}

        def state(n: int) -> dict:
            """h_n of this process's slabs (owned rows valid), replaying its checkpoint segment."""
            c = n // K
            if seg_cache["index"] != c:
                states = {c * K: ckpt[c]}
                cur = ckpt[c]
                for m in range(c * K, min(c * K + K, T) - 1):
                    nxt = {s: self._ext(s, self.dtype) for s in L}
                    for s in L:
                        self.ops[s].forward_step(cur[s], fields[m], nxt[s], None)
                    self.ring.exchange(nxt, G, self.rows)
                    states[m + 1] = nxt
                    cur = nxt
                seg_cache["index"], seg_cache["states"] = c, states
            return seg_cache["states"][n]

        w = {s: self._ext(s, self.dtype) for s in L}
        w_next = {s: self._ext(s, self.dtype) for s in L}
        slope = self._sums()
        grho = torch.empty(self.nx, dtype=self.dtype, device=self.device)
        g_H = torch.zeros(self.nx, dtype=self.dtype, device=self.device)

        def field_adj(n: int) -> None:
            """grho of step n and g_H += g_E_total of step n, from the gathered slope sums."""
            self.field_op.backward_field(self.ring.gather_rows(slope, self.rows), fields[n],
                                         None if gEh is None else gEh[n], None if gee is None else gee[n:n + 1],
                                         g_H, grho)

        g_ff = None if g_f_final_rows is None else self._place(g_f_final_rows, self.dtype)
        h_last = state(T - 1)
        for s in L:
            self.ops[s].backward_start(None if g_ff is None else g_ff[s], h_last[s], fields[T - 1], w[s], slope[s])
        del g_ff
        field_adj(T - 1)
        for n in range(T - 1, 0, -1):
            self.ring.exchange(w, G, self.rows)
            h_prev = state(n - 1)
            for s in L:
                self.ops[s].backward_step(w[s], None, grho, fields[n], fields[n - 1], h_prev[s], w_next[s], slope[s])
            field_adj(n - 1)
            w, w_next = w_next, w
        self.ring.exchange(w, G, self.rows)
        g_f_iv = {s: torch.empty((self.rows[s], self.nv), dtype=self.dtype, device=self.device) for s in L}
        for s in L:
            self.ops[s].backward_finish(w[s], grho, fields[0], g_f_iv[s])
        return {"g_f_iv": g_f_iv, "g_H": g_H, "E_hist": E_hist, "ee_hist": ee_hist}
