"""Device plan: one (mesh, dt, f_eq, dtype) bound to one CUDA device.

Wraps the C ABI's ``vp_plan`` and owns the caller-side device memory the ABI expects
(workspaces cached per step count, tapes allocated per forward call) as torch tensors, so that
all device memory goes through torch's caching allocator.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _capi

_DTYPES = {torch.float32: _capi.VP_F32, torch.float64: _capi.VP_F64}


def as_torch_dtype(dtype) -> torch.dtype:
    if dtype in (None, "float32", "f32", np.float32, torch.float32):
        return torch.float32
    if dtype in ("float64", "f64", np.float64, torch.float64):
        return torch.float64
    raise ValueError(f"dtype must be float32 or float64, got {dtype!r}")


def _stream_handle(device: torch.device) -> int:
    return int(torch.cuda.current_stream(device).cuda_stream)


class Plan:
    """A ``vp_plan`` plus its workspace cache."""

    def __init__(self, mesh, dt: float, f_eq: np.ndarray, dtype=torch.float32, device=None):
        if not torch.cuda.is_available():
            raise RuntimeError("warp_vp_solver_b200 needs a CUDA device (no CPU fallback)")
        self.lib = _capi.load()
        self.dtype = as_torch_dtype(dtype)
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None \
            else torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.nx, self.nv = int(mesh.nx), int(mesh.nv)
        self.dt = float(dt)
        f_eq = np.ascontiguousarray(np.asarray(f_eq, dtype=np.float64))
        # one row (nv,): an x-invariant f_eq given without its (nx, nv) array
        self.row_only = f_eq.shape == (self.nv,)
        if not self.row_only and f_eq.shape != (self.nx, self.nv):
            raise ValueError(f"f_eq shape {f_eq.shape} != ({self.nx}, {self.nv}) or ({self.nv},)")
        self.f_eq = f_eq
        self._xs = np.ascontiguousarray(np.asarray(mesh.xs, dtype=np.float64))
        self._vs = np.ascontiguousarray(np.asarray(mesh.vs, dtype=np.float64))
        desc = _capi.MeshDesc(self.nx, self.nv, _capi.dbl_ptr(self._xs), _capi.dbl_ptr(self._vs),
                              float(mesh.dx), float(mesh.dv), float(mesh.period_x),
                              float(mesh.period_v))
        handle = ctypes.c_void_p()
        create = self.lib.vp_plan_create_from_row if self.row_only else self.lib.vp_plan_create
        with torch.cuda.device(self.device):
            _capi.check(create(ctypes.byref(desc), self.dt, _capi.dbl_ptr(f_eq), _DTYPES[self.dtype],
                               ctypes.byref(handle)))
        self._h = handle
        self._ws: dict[tuple[int, int], torch.Tensor] = {}
        self._sizes: dict = {}   # checkpoint intervals and tape sizes per (n_steps, every), per launch shape

    # ---------------------------------------------------------------- housekeeping
    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.vp_plan_destroy(self._h)
            self._h = None
        self._ws = {}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def get_config(self) -> dict:
        c = _capi.LaunchConfig()
        _capi.check(self.lib.vp_plan_get_config(self._h, ctypes.byref(c)))
        return {f: getattr(c, f) for f, _ in _capi.LaunchConfig._fields_}

    def set_config(self, rows_per_cta: int | None = None, threads: int | None = None,
                   n_chunks: int | None = None, cluster_size: int | None = None,
                   stage_rows: int | None = None, stage_threads: int | None = None,
                   persist_rows: int | None = None, strip_rows: int | None = None,
                   strip_cols: int | None = None, strip_adj_cols: int | None = None) -> None:
        """Change the launch shape; arguments left as None keep their current values.
        ``stage_rows=0`` turns the staged forward step off, ``persist_rows=0`` the persistent
        (one launch per loop) path, ``strip_rows=0`` the strip (two launches per step) path;
        ``strip_cols`` / ``strip_adj_cols`` (128 or 256) set the columns a forward / adjoint strip
        CTA walks."""
        cur = self.get_config()
        c = _capi.LaunchConfig()
        c.rows_per_cta = cur["rows_per_cta"] if rows_per_cta is None else int(rows_per_cta)
        c.threads = cur["threads"] if threads is None else int(threads)
        c.n_chunks = cur["n_chunks"] if n_chunks is None else int(n_chunks)
        c.cluster_size = cur["cluster_size"] if cluster_size is None else int(cluster_size)
        c.stage_rows = cur["stage_rows"] if stage_rows is None else int(stage_rows)
        c.stage_threads = cur["stage_threads"] if stage_threads is None else int(stage_threads)
        c.persist_rows = cur["persist_rows"] if persist_rows is None else int(persist_rows)
        c.strip_rows = cur["strip_rows"] if strip_rows is None else int(strip_rows)
        c.strip_cols = 0 if strip_cols is None else int(strip_cols)
        c.strip_adj_cols = 0 if strip_adj_cols is None else int(strip_adj_cols)
        _capi.check(self.lib.vp_plan_set_config(self._h, ctypes.byref(c)))
        self._ws = {}   # workspace size depends on n_chunks and the persistent and strip launch shapes
        self._sizes = {}

    def set_wait_limit(self, ns: int) -> None:
        """Limit of each device-side grid-barrier wait of the persistent launches (ns; 0: no wait)."""
        _capi.check(self.lib.vp_plan_set_wait_limit(self._h, int(ns)))

    def status(self) -> int:
        """Device-side status flags (synchronous): VP_STATUS_NONFINITE_INPUT, VP_STATUS_WAIT_TIMEOUT."""
        f = ctypes.c_uint32()
        _capi.check(self.lib.vp_plan_status(self._h, ctypes.byref(f)))
        return int(f.value)

    def clear_status(self) -> None:
        _capi.check(self.lib.vp_plan_clear_status(self._h))

    def set_scheme(self, merged: bool) -> None:
        """Strang splitting (False) or the merged-Strang scheme of the reference's aggressive
        path (True)."""
        _capi.check(self.lib.vp_plan_set_scheme(
            self._h, _capi.VP_SCHEME_MERGED if merged else _capi.VP_SCHEME_STRANG))
        self._sizes = {}

    @property
    def merged(self) -> bool:
        out = ctypes.c_int32()
        _capi.check(self.lib.vp_plan_get_scheme(self._h, ctypes.byref(out)))
        return out.value == _capi.VP_SCHEME_MERGED

    def num_steps(self, t_final: float) -> int:
        out = ctypes.c_int32()
        _capi.check(self.lib.vp_num_steps(self._h, float(t_final), ctypes.byref(out)))
        return int(out.value)

    def resolve_every(self, n_steps: int, every: int | None) -> int:
        key = ("every", int(n_steps), int(every or 0))
        hit = self._sizes.get(key)
        if hit is None:
            out = ctypes.c_int32()
            _capi.check(self.lib.vp_resolve_checkpoint_every(self._h, int(n_steps), int(every or 0),
                                                             ctypes.byref(out)))
            hit = self._sizes[key] = int(out.value)
        return hit

    def workspace_bytes(self, n_steps: int, every: int) -> int:
        out = ctypes.c_size_t()
        _capi.check(self.lib.vp_workspace_bytes(self._h, int(n_steps), int(every), ctypes.byref(out)))
        return int(out.value)

    def tape_bytes(self, n_steps: int, every: int) -> int:
        key = ("tape", int(n_steps), int(every))
        hit = self._sizes.get(key)
        if hit is None:
            out = ctypes.c_size_t()
            _capi.check(self.lib.vp_tape_bytes(self._h, int(n_steps), int(every), ctypes.byref(out)))
            hit = self._sizes[key] = int(out.value)
        return hit

    def workspace(self, n_steps: int, every: int) -> torch.Tensor:
        key = (int(n_steps), int(every))
        ws = self._ws.get(key)
        if ws is None:
            nbytes = self.workspace_bytes(n_steps, every)
            ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=self.device)
            self._ws[key] = ws
        return ws

    # ---------------------------------------------------------------- tensors
    def to_f64(self, a) -> torch.Tensor:
        t = torch.as_tensor(a)
        return t.to(device=self.device, dtype=torch.float64).contiguous()

    def to_real(self, a) -> torch.Tensor:
        t = torch.as_tensor(a)
        return t.to(device=self.device, dtype=self.dtype).contiguous()

    # ---------------------------------------------------------------- forward / backward
    def forward(self, f_iv: torch.Tensor, H: torch.Tensor, n_steps: int, *, record_history: bool,
                want_tape: bool = False, checkpoint_every: int | None = None,
                want_f_final: bool = True):
        """Run ``n_steps`` Strang steps. Returns a dict of device tensors."""
        nx, nv, dev, dt = self.nx, self.nv, self.device, self.dtype
        f_iv = self.to_f64(f_iv).reshape(nx, nv)
        H = self.to_real(H).reshape(nx)
        every = self.resolve_every(n_steps, checkpoint_every)
        out = {
            "f_final": torch.empty((nx, nv), dtype=torch.float64, device=dev) if want_f_final else None,
            "f_hist": torch.empty((n_steps, nx, nv), dtype=dt, device=dev) if record_history else None,
            "E_hist": torch.empty((n_steps, nx), dtype=dt, device=dev),
            "ee_hist": torch.empty((n_steps,), dtype=dt, device=dev),
            "tape": None,
            "every": every,
        }
        if want_tape and n_steps > 0:
            out["tape"] = torch.empty(self.tape_bytes(n_steps, every), dtype=torch.uint8, device=dev)
        ws = self.workspace(n_steps, every)
        with torch.cuda.device(dev):
            _capi.check(self.lib.vp_forward(
                self._h, _capi.ptr(f_iv), _capi.ptr(H), int(n_steps),
                _capi.ptr(out["f_final"]), _capi.ptr(out["f_hist"]),
                _capi.ptr(out["E_hist"]) if n_steps > 0 else None,
                _capi.ptr(out["ee_hist"]) if n_steps > 0 else None,
                _capi.ptr(out["tape"]), int(every), _capi.ptr(ws), ws.numel(),
                _stream_handle(dev)))
        out["H"] = H
        return out

    def forward_stream_history(self, f_iv, H, n_steps: int, slots: int = 4, want_tape: bool = False,
                               checkpoint_every: int | None = None, want_f_final: bool = True):
        """Forward with f_hist streamed into a pinned host tensor through a ring of `slots`
        device buffers (vp_forward_stream_history). The host history is complete once the
        current stream is; the returned dict keeps the ring and copy stream alive."""
        nx, nv, dev, dt = self.nx, self.nv, self.device, self.dtype
        if n_steps < 1:
            raise ValueError("n_steps must be >= 1")
        f_iv = self.to_f64(f_iv).reshape(nx, nv)
        H = self.to_real(H).reshape(nx)
        every = self.resolve_every(n_steps, checkpoint_every)
        host = torch.empty((n_steps, nx, nv), dtype=dt, pin_memory=True)
        ring = torch.empty((slots, nx, nv), dtype=dt, device=dev)
        out = {
            "f_final": torch.empty((nx, nv), dtype=torch.float64, device=dev) if want_f_final else None,
            "f_hist": host,
            "E_hist": torch.empty((n_steps, nx), dtype=dt, device=dev),
            "ee_hist": torch.empty((n_steps,), dtype=dt, device=dev),
            "tape": torch.empty(self.tape_bytes(n_steps, every), dtype=torch.uint8, device=dev)
            if want_tape else None,
            "every": every,
        }
        ws = self.workspace(n_steps, every)
        with torch.cuda.device(dev):
            copy = torch.cuda.Stream(dev)
            _capi.check(self.lib.vp_forward_stream_history(
                self._h, _capi.ptr(f_iv), _capi.ptr(H), int(n_steps), _capi.ptr(out["f_final"]),
                host.data_ptr(), _capi.ptr(ring), int(slots), _capi.ptr(out["E_hist"]),
                _capi.ptr(out["ee_hist"]), _capi.ptr(out["tape"]), int(every), _capi.ptr(ws), ws.numel(),
                _stream_handle(dev), int(copy.cuda_stream)))
        out["H"] = H
        out["_ring"] = (ring, copy)
        return out

    def backward(self, H: torch.Tensor, n_steps: int, tape: torch.Tensor | None, every: int,
                 g_f_final=None, g_f_hist=None, g_E_hist=None, g_ee_hist=None):
        """Discrete adjoint. Cotangents are device tensors or None (zero)."""
        nx, nv, dev = self.nx, self.nv, self.device
        H = self.to_real(H).reshape(nx)

        def prep(g, shape):
            if g is None:
                return None
            return self.to_real(g).reshape(shape)

        g_ff = prep(g_f_final, (nx, nv))
        g_fh = prep(g_f_hist, (n_steps, nx, nv))
        g_Eh = prep(g_E_hist, (n_steps, nx))
        g_ee = prep(g_ee_hist, (n_steps,))
        g_fiv = torch.empty((nx, nv), dtype=self.dtype, device=dev)
        g_H = torch.empty((nx,), dtype=self.dtype, device=dev)
        ws = self.workspace(n_steps, every)
        with torch.cuda.device(dev):
            _capi.check(self.lib.vp_backward(
                self._h, _capi.ptr(H), int(n_steps), _capi.ptr(tape), int(every),
                _capi.ptr(g_ff), _capi.ptr(g_fh), _capi.ptr(g_Eh), _capi.ptr(g_ee),
                _capi.ptr(g_fiv), _capi.ptr(g_H), _capi.ptr(ws), ws.numel(), _stream_handle(dev)))
        return g_fiv, g_H

    # ---------------------------------------------------------------- single-stage operators
    def kl_divergence(self, f, eps: float = 1e-12, want_grad: bool = True):
        """KL(f || f_eq) over phase space and its gradient (float64 device tensors)."""
        f = self.to_f64(f).reshape(self.nx, self.nv)
        value = torch.empty(1, dtype=torch.float64, device=self.device)
        grad = torch.empty_like(f) if want_grad else None
        with torch.cuda.device(self.device):
            _capi.check(self.lib.vp_kl_divergence(self._h, _capi.ptr(f), float(eps), _capi.ptr(value),
                                                  _capi.ptr(grad), _stream_handle(self.device)))
        return value[0], grad

    def compute_rho(self, f) -> torch.Tensor:
        f = self.to_f64(f).reshape(self.nx, self.nv)
        rho = torch.empty(self.nx, dtype=self.dtype, device=self.device)
        with torch.cuda.device(self.device):
            _capi.check(self.lib.vp_compute_rho(self._h, _capi.ptr(f), _capi.ptr(rho),
                                                _stream_handle(self.device)))
        return rho

    def poisson(self, x, adjoint: bool = False) -> torch.Tensor:
        x = self.to_real(x).reshape(self.nx)
        out = torch.empty_like(x)
        with torch.cuda.device(self.device):
            _capi.check(self.lib.vp_poisson(self._h, _capi.ptr(x), _capi.ptr(out), int(adjoint),
                                            _stream_handle(self.device)))
        return out

    def electric_energy(self, E) -> torch.Tensor:
        E = self.to_real(E).reshape(self.nx)
        ee = torch.empty(1, dtype=self.dtype, device=self.device)
        with torch.cuda.device(self.device):
            _capi.check(self.lib.vp_electric_energy(self._h, _capi.ptr(E), _capi.ptr(ee),
                                                    _stream_handle(self.device)))
        return ee

    def semilag_x(self, a, dt: float, adjoint: bool = False) -> torch.Tensor:
        a = self.to_real(a).reshape(self.nx, self.nv)
        out = torch.empty_like(a)
        with torch.cuda.device(self.device):
            _capi.check(self.lib.vp_semilag_x(self._h, _capi.ptr(a), _capi.ptr(out), float(dt),
                                              int(adjoint), _stream_handle(self.device)))
        return out

    def semilag_v(self, a, E_total, dt: float, adjoint: bool = False, f_in=None):
        a = self.to_real(a).reshape(self.nx, self.nv)
        Et = self.to_real(E_total).reshape(self.nx)
        out = torch.empty_like(a)
        g_E = None
        f_t = None
        if adjoint and f_in is not None:
            f_t = self.to_real(f_in).reshape(self.nx, self.nv)
            g_E = torch.empty(self.nx, dtype=self.dtype, device=self.device)
        with torch.cuda.device(self.device):
            _capi.check(self.lib.vp_semilag_v(self._h, _capi.ptr(a), _capi.ptr(Et), _capi.ptr(out),
                                              float(dt), int(adjoint), _capi.ptr(f_t), _capi.ptr(g_E),
                                              _stream_handle(self.device)))
        return (out, g_E) if adjoint else out
