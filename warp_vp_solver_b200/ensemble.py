"""Ensembles: many uneven instances advanced together, one persistent launch per time step.

Each instance has its own mesh (nx, nv, lengths), time step, equilibrium ``f_eq``, initial
state and external field ``H``; all share the number of steps. The numerics of every instance
are exactly those of :class:`WarpVlasovPoissonSolver` (the reference's ``run_forward`` loop,
warp_vp_solver/solver.py:742-1105, and its adjoint, solver.py:418-612); what changes is the
schedule: the C ABI's ``vp_batch_*`` entry points sweep the tiles of all instances (sorted
longest first) with one persistent grid, and each instance's field solve runs in the CTA that
finishes its last tile.

Device arrays are PACKED: instance ``i``'s (nx_i, nv_i) block of a cell array starts at cell
offset ``cell_offsets[i]``, its nx_i row block at ``row_offsets[i]``; per-step histories are
``(n_steps, nx_i)`` blocks at ``n_steps * row_offsets[i]`` and ``ee`` entries at
``i * n_steps``. :meth:`Ensemble.pack_cells` / :meth:`Ensemble.unpack` convert.
"""

from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np
import torch

from . import _capi
from .plan import _DTYPES, _stream_handle, as_torch_dtype


def packed_offsets(shapes: Sequence[tuple[int, int]]):
    """Cell and row offsets of the packed layout (instances in the given order)."""
    cells = np.zeros(len(shapes), dtype=np.int64)
    rows = np.zeros(len(shapes), dtype=np.int64)
    c = r = 0
    for i, (nx, nv) in enumerate(shapes):
        cells[i], rows[i] = c, r
        c += int(nx) * int(nv)
        r += int(nx)
    return cells, rows, c, r


class Ensemble:
    """A ``vp_batch``: instances bound to one CUDA device, plus a workspace cache."""

    def __init__(self, meshes: Sequence, dts, f_eqs: Sequence, dtype=torch.float32, device=None):
        if not torch.cuda.is_available():
            raise RuntimeError("warp_vp_solver_b200 needs a CUDA device (no CPU fallback)")
        n = len(meshes)
        if n < 1:
            raise ValueError("an ensemble needs at least one instance")
        dts = np.broadcast_to(np.asarray(dts, dtype=np.float64), (n,)).copy()
        if len(f_eqs) != n:
            raise ValueError(f"{len(f_eqs)} f_eq arrays for {n} meshes")
        self.lib = _capi.load()
        self.dtype = as_torch_dtype(dtype)
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None \
            else torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.n = n
        self.meshes = list(meshes)
        self.dts = dts
        self.shapes = [(int(m.nx), int(m.nv)) for m in meshes]
        keep = []
        descs = (_capi.MeshDesc * n)()
        feq_ptrs = (ctypes.POINTER(ctypes.c_double) * n)()
        for i, (m, fe) in enumerate(zip(meshes, f_eqs)):
            xs = np.ascontiguousarray(np.asarray(m.xs, dtype=np.float64))
            vs = np.ascontiguousarray(np.asarray(m.vs, dtype=np.float64))
            fe = np.ascontiguousarray(np.asarray(fe, dtype=np.float64))
            if fe.shape != self.shapes[i]:
                raise ValueError(f"instance {i}: f_eq shape {fe.shape} != {self.shapes[i]}")
            keep += [xs, vs, fe]
            descs[i] = _capi.MeshDesc(int(m.nx), int(m.nv), _capi.dbl_ptr(xs), _capi.dbl_ptr(vs),
                                      float(m.dx), float(m.dv), float(m.period_x), float(m.period_v))
            feq_ptrs[i] = _capi.dbl_ptr(fe)
        handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _capi.check(self.lib.vp_batch_create(int(n), descs, _capi.dbl_ptr(dts), feq_ptrs,
                                                 _DTYPES[self.dtype], ctypes.byref(handle)))
        self._h = handle
        tc, tr = ctypes.c_int64(), ctypes.c_int64()
        co = np.zeros(n, dtype=np.int64)
        ro = np.zeros(n, dtype=np.int64)
        _capi.check(self.lib.vp_batch_offsets(
            self._h, ctypes.byref(tc), ctypes.byref(tr),
            co.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
            ro.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
        self.cell_offsets, self.row_offsets = co, ro
        self.total_cells, self.total_rows = int(tc.value), int(tr.value)
        self._ws: dict[int, torch.Tensor] = {}

    # ---------------------------------------------------------------- housekeeping
    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.vp_batch_destroy(self._h)
            self._h = None
        self._ws = {}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_config(self) -> dict:
        c = _capi.BatchConfig()
        _capi.check(self.lib.vp_batch_get_config(self._h, ctypes.byref(c)))
        return {f: getattr(c, f) for f, _ in _capi.BatchConfig._fields_}

    def set_config(self, rows_per_tile: int | None = None, chunk_cols: int | None = None,
                   threads: int | None = None, ctas_per_sm: int | None = None,
                   strip: int | None = None) -> None:
        """Change the tile shape (None keeps the current value); ``strip=1`` runs the steps on the
        strip kernels (where every instance qualifies), ``strip=0`` on the tile kernels.
        Invalidates captured graphs."""
        cur = self.get_config()
        c = _capi.BatchConfig()
        c.rows_per_tile = cur["rows_per_tile"] if rows_per_tile is None else int(rows_per_tile)
        c.chunk_cols = cur["chunk_cols"] if chunk_cols is None else int(chunk_cols)
        c.threads = cur["threads"] if threads is None else int(threads)
        c.ctas_per_sm = cur["ctas_per_sm"] if ctas_per_sm is None else int(ctas_per_sm)
        c.strip = cur["strip"] if strip is None else int(strip)
        with torch.cuda.device(self.device):
            _capi.check(self.lib.vp_batch_set_config(self._h, ctypes.byref(c)))
        self._ws = {}

    @property
    def cells_per_step(self) -> int:
        return self.total_cells

    def num_steps(self, t_final: float) -> int:
        """Common step count: ``int(t_final / dt)`` must agree across instances."""
        steps = {int(float(t_final) / float(dt)) for dt in self.dts}
        if len(steps) != 1:
            raise ValueError(f"instances disagree on the number of steps for t_final={t_final}: "
                             f"{sorted(steps)}")
        return steps.pop()

    def workspace_bytes(self, n_steps: int) -> int:
        out = ctypes.c_size_t()
        _capi.check(self.lib.vp_batch_workspace_bytes(self._h, int(n_steps), ctypes.byref(out)))
        return int(out.value)

    def tape_bytes(self, n_steps: int) -> int:
        out = ctypes.c_size_t()
        _capi.check(self.lib.vp_batch_tape_bytes(self._h, int(n_steps), ctypes.byref(out)))
        return int(out.value)

    def workspace(self, n_steps: int) -> torch.Tensor:
        ws = self._ws.get(int(n_steps))
        if ws is None:
            ws = torch.empty(max(self.workspace_bytes(n_steps), 256), dtype=torch.uint8,
                             device=self.device)
            self._ws[int(n_steps)] = ws
        return ws

    # ---------------------------------------------------------------- packing
    def pack_cells(self, arrays, dtype=torch.float64) -> torch.Tensor:
        out = torch.empty(self.total_cells, dtype=dtype, device=self.device)
        for i, a in enumerate(arrays):
            nx, nv = self.shapes[i]
            o = int(self.cell_offsets[i])
            out[o:o + nx * nv] = torch.as_tensor(a).to(device=self.device, dtype=dtype).reshape(-1)
        return out

    def pack_rows(self, arrays, dtype=None) -> torch.Tensor:
        dtype = self.dtype if dtype is None else dtype
        out = torch.empty(self.total_rows, dtype=dtype, device=self.device)
        for i, a in enumerate(arrays):
            nx = self.shapes[i][0]
            o = int(self.row_offsets[i])
            out[o:o + nx] = torch.as_tensor(a).to(device=self.device, dtype=dtype).reshape(-1)
        return out

    def pack_hist(self, arrays, n_steps: int) -> torch.Tensor:
        out = torch.empty(n_steps * self.total_rows, dtype=self.dtype, device=self.device)
        for i, a in enumerate(arrays):
            nx = self.shapes[i][0]
            o = n_steps * int(self.row_offsets[i])
            out[o:o + n_steps * nx] = torch.as_tensor(a).to(device=self.device,
                                                            dtype=self.dtype).reshape(-1)
        return out

    def cells_of(self, packed: torch.Tensor, i: int) -> torch.Tensor:
        nx, nv = self.shapes[i]
        o = int(self.cell_offsets[i])
        return packed[o:o + nx * nv].view(nx, nv)

    def rows_of(self, packed: torch.Tensor, i: int) -> torch.Tensor:
        nx = self.shapes[i][0]
        o = int(self.row_offsets[i])
        return packed[o:o + nx]

    def hist_of(self, packed: torch.Tensor, i: int, n_steps: int) -> torch.Tensor:
        nx = self.shapes[i][0]
        o = n_steps * int(self.row_offsets[i])
        return packed[o:o + n_steps * nx].view(n_steps, nx)

    def ee_of(self, packed: torch.Tensor, i: int, n_steps: int) -> torch.Tensor:
        return packed[i * n_steps:(i + 1) * n_steps]

    # ---------------------------------------------------------------- forward / backward
    def alloc_outputs(self, n_steps: int, want_tape: bool = False, want_f_final: bool = True):
        dev, dt = self.device, self.dtype
        return {
            "f_final": torch.empty(self.total_cells, dtype=torch.float64, device=dev)
            if want_f_final else None,
            "E_hist": torch.empty(n_steps * self.total_rows, dtype=dt, device=dev),
            "ee_hist": torch.empty(n_steps * self.n, dtype=dt, device=dev),
            "tape": torch.empty(self.tape_bytes(n_steps), dtype=torch.uint8, device=dev)
            if want_tape else None,
        }

    def forward_into(self, f_iv: torch.Tensor, H: torch.Tensor, n_steps: int, out: dict) -> None:
        """Launch the forward loop into preallocated packed buffers (capture-safe)."""
        ws = self.workspace(n_steps)
        _capi.check(self.lib.vp_batch_forward(
            self._h, _capi.ptr(f_iv), _capi.ptr(H), int(n_steps), _capi.ptr(out["f_final"]),
            _capi.ptr(out["E_hist"]), _capi.ptr(out["ee_hist"]), _capi.ptr(out["tape"]),
            _capi.ptr(ws), ws.numel(), _stream_handle(self.device)))

    def backward_into(self, H: torch.Tensor, n_steps: int, tape: torch.Tensor, g_f_final,
                      g_E_hist, g_ee_hist, g_f_iv: torch.Tensor, g_H: torch.Tensor) -> None:
        """Launch the adjoint loop into preallocated packed buffers (capture-safe)."""
        ws = self.workspace(n_steps)
        _capi.check(self.lib.vp_batch_backward(
            self._h, _capi.ptr(H), int(n_steps), _capi.ptr(tape), _capi.ptr(g_f_final),
            _capi.ptr(g_E_hist), _capi.ptr(g_ee_hist), _capi.ptr(g_f_iv), _capi.ptr(g_H),
            _capi.ptr(ws), ws.numel(), _stream_handle(self.device)))

    def forward(self, f_iv, H, n_steps: int, want_tape: bool = False, want_f_final: bool = True):
        """Packed forward: f_iv (total_cells,) float64, H (total_rows,) of the ensemble dtype."""
        if n_steps < 1:
            raise ValueError("ensembles need n_steps >= 1")
        f_iv = torch.as_tensor(f_iv).to(device=self.device, dtype=torch.float64).contiguous()
        H = torch.as_tensor(H).to(device=self.device, dtype=self.dtype).contiguous()
        if f_iv.numel() != self.total_cells or H.numel() != self.total_rows:
            raise ValueError(f"packed f_iv must have {self.total_cells} cells and H "
                             f"{self.total_rows} rows (got {f_iv.numel()}, {H.numel()})")
        out = self.alloc_outputs(n_steps, want_tape, want_f_final)
        with torch.cuda.device(self.device):
            self.forward_into(f_iv, H, n_steps, out)
        out["H"] = H
        return out

    def backward(self, H, n_steps: int, tape: torch.Tensor, g_f_final=None, g_E_hist=None,
                 g_ee_hist=None):
        """Packed adjoint; cotangents are packed tensors or None (zero)."""
        H = torch.as_tensor(H).to(device=self.device, dtype=self.dtype).contiguous()

        def prep(g, n):
            if g is None:
                return None
            g = torch.as_tensor(g).to(device=self.device, dtype=self.dtype).contiguous()
            if g.numel() != n:
                raise ValueError(f"packed cotangent has {g.numel()} entries, {n} expected")
            return g

        g_ff = prep(g_f_final, self.total_cells)
        g_Eh = prep(g_E_hist, n_steps * self.total_rows)
        g_ee = prep(g_ee_hist, n_steps * self.n)
        g_fiv = torch.empty(self.total_cells, dtype=self.dtype, device=self.device)
        g_H = torch.empty(self.total_rows, dtype=self.dtype, device=self.device)
        with torch.cuda.device(self.device):
            self.backward_into(H, n_steps, tape, g_ff, g_Eh, g_ee, g_fiv, g_H)
        return g_fiv, g_H

    # ---------------------------------------------------------------- list front end
    def run_forward(self, f_ivs, Hs, t_final: float):
        """Per-instance ``(f_final, None, E_hist, ee_hist)`` tuples (as ``run_forward`` returns
        with ``record_history=False``), as numpy arrays."""
        T = self.num_steps(t_final)
        out = self.forward(self.pack_cells(f_ivs), self.pack_rows(Hs), T)
        res = []
        for i in range(self.n):
            res.append((self.cells_of(out["f_final"], i).cpu().numpy(), None,
                        self.hist_of(out["E_hist"], i, T).cpu().numpy(),
                        self.ee_of(out["ee_hist"], i, T).cpu().numpy()))
        return res

    def run_forward_torch(self, f_iv: torch.Tensor, H: torch.Tensor, n_steps: int):
        """Differentiable packed forward: returns packed (f_final, E_hist, ee_hist)."""
        return _EnsembleFunction.apply(f_iv, H, self, int(n_steps))

    def capture(self, n_steps: int, adjoint: bool = True) -> "EnsembleGraph":
        return EnsembleGraph(self, n_steps, adjoint)


class _EnsembleFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, f_iv, H, ens: Ensemble, n_steps: int):
        out = ens.forward(f_iv.detach(), H.detach(), n_steps, want_tape=True)
        ctx.ens = ens
        ctx.n_steps = n_steps
        ctx.f_dtype, ctx.f_device = f_iv.dtype, f_iv.device
        ctx.H_dtype, ctx.H_device = H.dtype, H.device
        ctx.save_for_backward(out["H"], out["tape"])
        return out["f_final"], out["E_hist"], out["ee_hist"]

    @staticmethod
    def backward(ctx, g_f_final, g_E_hist, g_ee_hist):
        H, tape = ctx.saved_tensors
        g_fiv, g_H = ctx.ens.backward(H, ctx.n_steps, tape, g_f_final, g_E_hist, g_ee_hist)
        return (g_fiv.to(device=ctx.f_device, dtype=ctx.f_dtype),
                g_H.to(device=ctx.H_device, dtype=ctx.H_dtype), None, None)


class EnsembleGraph:
    """The whole ensemble time loop (forward, and optionally the adjoint of a cost whose
    cotangents are written into ``g_ee_hist`` / ``g_E_hist`` / ``g_f_final``) captured once as
    a CUDA graph over static packed buffers; :meth:`replay` relaunches it.

    Inputs to fill before ``replay``: ``f_iv`` (float64 cells), ``H`` (rows), and for the
    adjoint the cotangent buffers. Outputs: ``out["f_final"|"E_hist"|"ee_hist"]``, ``g_f_iv``,
    ``g_H``."""

    def __init__(self, ens: Ensemble, n_steps: int, adjoint: bool = True):
        if n_steps < 1:
            raise ValueError("ensembles need n_steps >= 1")
        self.ens, self.n_steps, self.adjoint = ens, int(n_steps), bool(adjoint)
        dev, dt = ens.device, ens.dtype
        self.f_iv = torch.zeros(ens.total_cells, dtype=torch.float64, device=dev)
        self.H = torch.zeros(ens.total_rows, dtype=dt, device=dev)
        self.out = ens.alloc_outputs(self.n_steps, want_tape=adjoint)
        self.g_f_final = torch.zeros(ens.total_cells, dtype=dt, device=dev) if adjoint else None
        self.g_E_hist = torch.zeros(self.n_steps * ens.total_rows, dtype=dt, device=dev) \
            if adjoint else None
        self.g_ee_hist = torch.zeros(self.n_steps * ens.n, dtype=dt, device=dev) if adjoint else None
        self.g_f_iv = torch.empty(ens.total_cells, dtype=dt, device=dev) if adjoint else None
        self.g_H = torch.empty(ens.total_rows, dtype=dt, device=dev) if adjoint else None
        ens.workspace(self.n_steps)
        with torch.cuda.device(dev):
            side = torch.cuda.Stream(dev)
            side.wait_stream(torch.cuda.current_stream(dev))
            with torch.cuda.stream(side):
                self._launch()          # warm-up outside capture (first-use attribute setup)
            torch.cuda.current_stream(dev).wait_stream(side)
            torch.cuda.synchronize(dev)
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.graph):
                self._launch()

    def _launch(self) -> None:
        e, T = self.ens, self.n_steps
        e.forward_into(self.f_iv, self.H, T, self.out)
        if self.adjoint:
            e.backward_into(self.H, T, self.out["tape"], self.g_f_final, self.g_E_hist,
                            self.g_ee_hist, self.g_f_iv, self.g_H)

    def replay(self) -> None:
        self.graph.replay()
