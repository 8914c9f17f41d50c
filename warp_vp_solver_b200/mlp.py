"""Tensor-core MLP (the surrogate's network) over the ``vp_mlp_*`` C ABI.

BF16 operands with FP32 accumulation on the tcgen05 tensor cores, FP32 master weights, Adam with
its step count on the device (so a whole training step can be captured in a CUDA graph). There is
no CPU fallback.
"""

from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np
import torch

from . import _capi
from .plan import _stream_handle


def init_params(widths: Sequence[int], seed: int) -> np.ndarray:
    """U(-1/sqrt(fan_in), 1/sqrt(fan_in)) for weights and biases (the torch.nn.Linear default),
    packed per layer as W_l [out, in] row-major then b_l."""
    rng = np.random.default_rng(seed)
    chunks = []
    for i in range(len(widths) - 1):
        k, n = widths[i], widths[i + 1]
        a = 1.0 / np.sqrt(k)
        chunks += [rng.uniform(-a, a, n * k), rng.uniform(-a, a, n)]
    return np.concatenate(chunks).astype(np.float32)


class MLP:
    """widths[0] -> ... -> widths[-1], GELU between layers."""

    def __init__(self, widths: Sequence[int], max_batch: int, seed: int = 0, device=None):
        if not torch.cuda.is_available():
            raise RuntimeError("warp_vp_solver_b200 needs a CUDA device (no CPU fallback)")
        self.lib = _capi.load()
        self.widths = [int(w) for w in widths]
        self.max_batch = int(max_batch)
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None \
            else torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        w = (ctypes.c_int32 * len(self.widths))(*self.widths)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _capi.check(self.lib.vp_mlp_create(len(self.widths) - 1, w, self.max_batch, ctypes.byref(h)))
        self._h = h
        n = ctypes.c_int64()
        _capi.check(self.lib.vp_mlp_param_count(self._h, ctypes.byref(n)))
        self.n_params = int(n.value)
        self._loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        self.set_params(init_params(self.widths, seed))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.vp_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _s(self) -> int:
        return _stream_handle(self.device)

    def _f32(self, a) -> torch.Tensor:
        return torch.as_tensor(a).to(device=self.device, dtype=torch.float32).contiguous()

    # ---------------------------------------------------------------- parameters
    def set_params(self, params) -> None:
        p = self._f32(params).reshape(-1)
        if p.numel() != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters, got {p.numel()}")
        with torch.cuda.device(self.device):
            _capi.check(self.lib.vp_mlp_set_params(self._h, _capi.ptr(p), self._s()))
        torch.cuda.current_stream(self.device).synchronize()

    def get_params(self) -> torch.Tensor:
        p = torch.empty(self.n_params, dtype=torch.float32, device=self.device)
        _capi.check(self.lib.vp_mlp_get_params(self._h, _capi.ptr(p), None, self._s()))
        return p

    def get_grads(self) -> torch.Tensor:
        g = torch.empty(self.n_params, dtype=torch.float32, device=self.device)
        _capi.check(self.lib.vp_mlp_get_params(self._h, None, _capi.ptr(g), self._s()))
        return g

    # ---------------------------------------------------------------- compute
    def forward(self, X, rows=None, out: torch.Tensor | None = None) -> torch.Tensor:
        """Y = net(X[rows]) (rows optional int32 device indices)."""
        X = self._f32(X)
        M = int(rows.numel()) if rows is not None else int(X.shape[0])
        Y = out if out is not None else torch.empty((M, self.widths[-1]), dtype=torch.float32,
                                                    device=self.device)
        self.forward_into(X, rows, M, Y)
        return Y

    def forward_into(self, X: torch.Tensor, rows, M: int, Y: torch.Tensor | None) -> None:
        _capi.check(self.lib.vp_mlp_forward(
            self._h, _capi.ptr(X), int(X.stride(0)), _capi.ptr(rows), int(M), _capi.ptr(Y),
            int(Y.stride(0)) if Y is not None else 0, self._s()))

    def backward(self, g_Y, param_grads: bool = True, input_grad: bool = False):
        """Backward of the last forward; returns g_X when ``input_grad``."""
        g_Y = self._f32(g_Y)
        M = int(g_Y.shape[0])
        g_X = torch.empty((M, self.widths[0]), dtype=torch.float32, device=self.device) \
            if input_grad else None
        _capi.check(self.lib.vp_mlp_backward(
            self._h, _capi.ptr(g_Y), int(g_Y.stride(0)), M, int(bool(param_grads)), _capi.ptr(g_X),
            int(g_X.stride(0)) if g_X is not None else 0, self._s()))
        return g_X

    def backward_into(self, g_Y: torch.Tensor, g_X: torch.Tensor | None, param_grads: bool) -> None:
        """Capture-safe backward into preallocated tensors."""
        _capi.check(self.lib.vp_mlp_backward(
            self._h, _capi.ptr(g_Y), int(g_Y.stride(0)), int(g_Y.shape[0]), int(bool(param_grads)),
            _capi.ptr(g_X), int(g_X.stride(0)) if g_X is not None else 0, self._s()))

    def mse_backward_into(self, T: torch.Tensor, rows, M: int, loss: torch.Tensor | None) -> None:
        _capi.check(self.lib.vp_mlp_mse_backward(self._h, _capi.ptr(T), int(T.stride(0)),
                                                 _capi.ptr(rows), int(M), _capi.ptr(loss), self._s()))

    def adam(self, lr: float = 1e-3, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8) -> None:
        _capi.check(self.lib.vp_mlp_adam(self._h, float(lr), float(beta1), float(beta2), float(eps),
                                         self._s()))

    def status(self) -> int:
        """Status flags (synchronous): bit 0 set when a tensor-core wait gave up."""
        f = ctypes.c_uint32()
        _capi.check(self.lib.vp_mlp_status(self._h, ctypes.byref(f)))
        return int(f.value)

    def clear_status(self) -> None:
        _capi.check(self.lib.vp_mlp_clear_status(self._h))

    def set_wait_limit(self, ns: int) -> None:
        """Limit of each bounded tensor-core wait in nanoseconds (default 1 s; 0: one poll)."""
        _capi.check(self.lib.vp_mlp_set_wait_limit(self._h, int(ns)))

    def train_step(self, X, T, rows=None) -> torch.Tensor:
        """forward + mean-squared-error backward (no Adam); returns the loss (device scalar)."""
        X, T = self._f32(X), self._f32(T)
        M = int(rows.numel()) if rows is not None else int(X.shape[0])
        self.forward_into(X, rows, M, None)
        self.mse_backward_into(T, rows, M, self._loss)
        return self._loss

    def fit(self, X, T, steps: int, batch: int, lr: float = 1e-3, seed: int = 0,
            use_graph: bool = True) -> np.ndarray:
        """Adam on the mean-squared error over minibatches drawn without replacement each epoch
        (indices precomputed on the host). One step = forward, loss backward, Adam; the step is
        captured once as a CUDA graph and replayed. Returns the loss history (float32)."""
        X, T = self._f32(X), self._f32(T)
        n = int(X.shape[0])
        batch = int(min(batch, n, self.max_batch))
        rng = np.random.default_rng(seed)
        per_epoch = n // batch
        n_epochs = (steps + per_epoch - 1) // per_epoch
        idx = np.concatenate([rng.permutation(n)[:per_epoch * batch] for _ in range(n_epochs)])
        idx = torch.tensor(idx[:steps * batch].reshape(steps, batch), dtype=torch.int32,
                           device=self.device)
        rows = torch.empty(batch, dtype=torch.int32, device=self.device)
        losses = torch.empty(steps, dtype=torch.float32, device=self.device)
        loss = torch.zeros(1, dtype=torch.float32, device=self.device)

        def step():
            self.forward_into(X, rows, batch, None)
            self.mse_backward_into(T, rows, batch, loss)
            self.adam(lr)

        graph = None
        if use_graph:
            with torch.cuda.device(self.device):
                rows.copy_(idx[0])
                # one eager forward/backward (no Adam) sets the kernels' attributes before capture
                self.forward_into(X, rows, batch, None)
                self.mse_backward_into(T, rows, batch, loss)
                torch.cuda.synchronize(self.device)
                graph = torch.cuda.CUDAGraph()
                with torch.cuda.graph(graph):
                    step()
        for i in range(steps):
            rows.copy_(idx[i])
            if graph is not None:
                graph.replay()
            else:
                step()
            losses[i:i + 1].copy_(loss)
        return losses.cpu().numpy()
