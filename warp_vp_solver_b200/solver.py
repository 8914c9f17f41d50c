"""Drop-in ``WarpVlasovPoissonSolver`` backed by the sm_100a kernels.

Same constructor, the same ``run_forward(f_iv, H, t_final, *, record_history)`` ->
``(f_final, f_hist, E_hist, ee_hist)`` contract, the same helper methods and the same error
messages as ``warp_vp_solver/solver.py`` (Forgotten/warp_vp_solver). The JAX ``custom_vjp``
front door (``run_forward_jax``, ``solver.py:1344-1407``) becomes ``run_forward_torch``, a
``torch.autograd.Function`` whose backward is the hand-written discrete adjoint kernel with
checkpointing and recomputation instead of a stored f history.

Array conventions: NumPy in, NumPy float64 out (like the reference); torch in, torch out on the
solver's device. The compute type is float32 by default (``dtype=torch.float64`` is available);
``f_final`` is always returned in float64 because it is formed as f_eq + delta in float64.
"""

from __future__ import annotations

from typing import Callable

import numpy as np
import torch

from .mesh import Mesh
from .plan import Plan, as_torch_dtype


class WarpVlasovPoissonSolver:
    """Vlasov-Poisson semi-Lagrangian solver on B200 (reference: solver.py:79-206)."""

    mesh: Mesh
    dt: float
    f_eq: np.ndarray

    _AGGRESSIVE_LAYOUTS = ("cpu_fused", "gpu_safe", "tiled")

    def __init__(
        self,
        mesh: Mesh,
        dt: float,
        f_eq: np.ndarray,
        *,
        optimized: bool = True,
        aggressive: bool = False,
        aggressive_layout: str = "cpu_fused",
        aggressive_tile_size: int = 32,
        record_history: bool = True,
        dtype=torch.float32,
        checkpoint_every: int | None = None,
        device=None,
    ):
        """Validate like the reference (solver.py:141-167), then bind lazily to a CUDA device.

        ``optimized=False`` and ``True`` run the same kernels (the reference's two paths are
        bit-identical, tests/test_optimized.py:163-181); ``optimized=False`` keeps the
        reference's refusal of ``record_history=False``. ``aggressive=True`` selects the
        merged-Strang scheme of the reference's aggressive path (any layout; one arithmetic chain).
        ``record_history`` sets the default of ``run_forward``'s keyword of the same name.
        ``checkpoint_every`` is the interval of the delta-f checkpoints the adjoint recomputes
        from; None keeps every step when that tape is at most 256 MiB and otherwise checkpoints
        every ceil(sqrt(n_steps)) steps.
        """
        self.mesh = mesh
        self.history_on_host = None   # None: stream f_hist to pinned host memory when > 256 MiB
        self.dt = float(dt)
        self.f_eq = np.asarray(f_eq, dtype=np.float64)
        if self.f_eq.shape != (mesh.nx, mesh.nv):
            raise ValueError(f"f_eq shape {self.f_eq.shape} != ({mesh.nx}, {mesh.nv})")
        _check_finite_host("f_eq", self.f_eq)
        self.optimized = bool(optimized)
        self.aggressive = bool(aggressive)
        if self.aggressive and not self.optimized:
            raise ValueError(
                "aggressive=True requires optimized=True - the aggressive "
                "path is built on top of the optimized buffers and fused-v "
                "kernel."
            )
        if aggressive_layout not in self._AGGRESSIVE_LAYOUTS:
            raise ValueError(
                f"aggressive_layout must be one of "
                f"{self._AGGRESSIVE_LAYOUTS!r}; got {aggressive_layout!r}."
            )
        self.aggressive_layout = aggressive_layout
        self.aggressive_tile_size = int(aggressive_tile_size)
        if self.aggressive_tile_size <= 0:
            raise ValueError(
                f"aggressive_tile_size must be positive; "
                f"got {aggressive_tile_size}."
            )
        self.record_history = bool(record_history)
        self.dtype = as_torch_dtype(dtype)
        if checkpoint_every is not None and int(checkpoint_every) < 0:
            raise ValueError(f"checkpoint_every must be >= 0; got {checkpoint_every}.")
        self.checkpoint_every = None if checkpoint_every is None else int(checkpoint_every)
        self._device = device
        self._plan: Plan | None = None
        self._torch_callable: Callable | None = None

    # ------------------------------------------------------------------ plumbing
    @property
    def plan(self) -> Plan:
        if self._plan is None:
            self._plan = Plan(self.mesh, self.dt, self.f_eq, dtype=self.dtype, device=self._device)
            if self.aggressive:
                self._plan.set_scheme(True)
        return self._plan

    @property
    def device(self) -> torch.device:
        return self.plan.device

    def num_steps(self, t_final: float) -> int:
        """int(t_final / dt) (solver.py:212-213)."""
        return int(t_final / self.dt)

    # ------------------------------------------------------------------ single-stage helpers
    def compute_rho(self, f):
        """rho(x) = integral (f_eq - f) dv by the trapezoidal rule (solver.py:393-397)."""
        rho = self.plan.compute_rho(f)
        return rho if isinstance(f, torch.Tensor) else rho.double().cpu().numpy()

    def compute_E_from_rho(self, rho):
        """Spectral Poisson solve of rho on the device (solver.py:399-404)."""
        E = self.plan.poisson(rho)
        return E if isinstance(rho, torch.Tensor) else E.double().cpu().numpy()

    def compute_E(self, f):
        """compute_E_from_rho(compute_rho(f)) (solver.py:406-407)."""
        return self.compute_E_from_rho(self.compute_rho(f))

    def compute_electric_energy(self, E) -> float:
        """0.5 * integral E^2 dx by the trapezoidal rule (solver.py:409-412)."""
        return float(self.plan.electric_energy(E).double().cpu()[0])

    # ------------------------------------------------------------------ forward
    def autotune(self, steps: int = 8, force: bool = False, cache_path: str | None = None) -> dict:
        """Time the candidate launch shapes on this solver's grid and keep the fastest (cached
        per device and shape; see ``warp_vp_solver_b200.autotune``)."""
        from .autotune import TuneCache, tune_plan
        return tune_plan(self.plan, steps=steps, force=force, cache=TuneCache(cache_path))

    def run_forward(self, f_iv, H, t_final: float, *, record_history: bool | None = None):
        """Strang-split time loop (solver.py:418-464).

        Returns ``(f_final, f_hist, E_hist, ee_hist)``: ``f_hist`` is None when
        ``record_history`` is False; ``E_hist`` holds E + H; ``ee_hist`` holds
        0.5*trapz(E^2)*dx of the self-consistent E (without H).
        """
        if record_history is None:
            record_history = self.record_history
        if not self.optimized and not record_history:
            raise ValueError(
                "record_history=False is only supported when the solver was "
                "constructed with optimized=True."
            )
        _check_finite_host("f_iv", f_iv)
        _check_finite_host("H", H)
        T = self.num_steps(t_final)
        as_torch = isinstance(f_iv, torch.Tensor)
        itemsize = 8 if self.dtype == torch.float64 else 4
        host_hist = self.history_on_host
        if host_hist is None:   # stream large histories to host memory instead of holding them
            host_hist = T * self.mesh.nx * self.mesh.nv * itemsize > (256 << 20)
        if record_history and not as_torch and host_hist and T >= 2:
            out = self.plan.forward_stream_history(f_iv, H, T)
            torch.cuda.current_stream(self.plan.device).synchronize()
        else:
            out = self.plan.forward(f_iv, H, T, record_history=record_history)
        res = (out["f_final"], out["f_hist"], out["E_hist"], out["ee_hist"])
        if as_torch:
            return res
        return tuple(None if r is None else r.double().cpu().numpy() for r in res)

    # ------------------------------------------------------------------ backward
    def _run_backward(self, f_iv, H, t_final, f_hist, g_f_final, g_f_hist, g_E_hist, g_ee_hist):
        """Discrete adjoint returning ``(g_f_iv, g_H)`` (solver.py:742-772).

        ``f_hist`` is accepted for signature compatibility and not read: the states the adjoint
        needs are recomputed on the device from checkpoints of a forward pass.
        """
        _check_finite_host("f_iv", f_iv)
        _check_finite_host("H", H)
        T = self.num_steps(t_final)
        as_torch = isinstance(f_iv, torch.Tensor)
        fwd = self.plan.forward(f_iv, H, T, record_history=False, want_tape=True,
                                checkpoint_every=self.checkpoint_every, want_f_final=False)
        g = self.plan.backward(fwd["H"], T, fwd["tape"], fwd["every"], g_f_final, g_f_hist,
                               g_E_hist, g_ee_hist)
        if as_torch:
            return g
        return tuple(x.double().cpu().numpy() for x in g)

    # ------------------------------------------------------------------ autograd front door
    @property
    def run_forward_torch(self) -> Callable:
        """``(f_iv, H, t_final) -> (f_final, f_hist, E_hist, ee_hist)`` with autograd.

        The torch counterpart of ``run_forward_jax`` (solver.py:1344-1407): gradients flow to
        ``f_iv`` and ``H``; ``t_final`` is static.
        """
        if self._torch_callable is None:
            solver = self

            def run(f_iv, H, t_final, *, record_history: bool | None = None):
                rh = solver.record_history if record_history is None else bool(record_history)
                if not solver.optimized and not rh:
                    raise ValueError(
                        "record_history=False is only supported when the solver was "
                        "constructed with optimized=True.")
                _check_finite_host("f_iv", f_iv)
                _check_finite_host("H", H)
                f_iv_t = f_iv if isinstance(f_iv, torch.Tensor) else torch.as_tensor(
                    np.asarray(f_iv, dtype=np.float64))
                H_t = H if isinstance(H, torch.Tensor) else torch.as_tensor(
                    np.asarray(H, dtype=np.float64))
                T = solver.num_steps(t_final)
                f_final, f_hist, E_hist, ee_hist = _VPFunction.apply(f_iv_t, H_t, solver, T, rh)
                return f_final, (f_hist if rh else None), E_hist, ee_hist

            self._torch_callable = run
        return self._torch_callable

    def check_status(self) -> None:
        """Raise if a kernel of this solver flagged a problem since the last check (synchronous):
        non-finite values in a device-resident f_iv or H (NumPy inputs are checked on the host
        before they are uploaded), or a bounded device-side wait that ran out. Clears the flags."""
        flags = self.plan.status()
        if flags:
            self.plan.clear_status()
        if flags & 1:
            raise ValueError("f_iv or H contains NaN or infinite values")
        if flags & 2:
            raise RuntimeError("a bounded device-side wait ran out; the last results are invalid")

    @property
    def run_forward_jax(self):
        raise NotImplementedError(
            "JAX is not part of this build; use run_forward_torch (a torch.autograd.Function "
            "with the same outputs and gradients)")


def _check_finite_host(name: str, a) -> None:
    """ValueError for NaN or infinite entries of a host (NumPy or CPU torch) input; device tensors
    are checked on the device (``check_status``) so that no call synchronises."""
    if isinstance(a, torch.Tensor):
        if a.device.type != "cpu":
            return
        ok = bool(torch.isfinite(a).all())
    else:
        ok = bool(np.isfinite(np.asarray(a, dtype=np.float64)).all())
    if not ok:
        raise ValueError(f"{name} contains NaN or infinite values")


class _VPFunction(torch.autograd.Function):
    """Forward: the fused time loop, writing a checkpoint tape. Backward: the fused adjoint."""

    @staticmethod
    def forward(ctx, f_iv, H, solver, n_steps, record_history):
        plan = solver.plan
        out = plan.forward(f_iv.detach(), H.detach(), n_steps, record_history=record_history,
                           want_tape=True, checkpoint_every=solver.checkpoint_every)
        # outputs the loss does not use arrive as None (no zero-filled cotangents to allocate,
        # fill and read in the adjoint)
        ctx.set_materialize_grads(False)
        ctx.plan = plan
        ctx.n_steps = n_steps
        ctx.every = out["every"]
        ctx.f_dtype = f_iv.dtype
        ctx.f_device = f_iv.device
        ctx.H_dtype = H.dtype
        ctx.H_device = H.device
        ctx.save_for_backward(out["H"], out["tape"] if out["tape"] is not None else
                              torch.empty(0, dtype=torch.uint8, device=plan.device))
        f_hist = out["f_hist"]
        if f_hist is None:
            f_hist = torch.empty((0,), dtype=plan.dtype, device=plan.device)
        return out["f_final"], f_hist, out["E_hist"], out["ee_hist"]

    @staticmethod
    def backward(ctx, g_f_final, g_f_hist, g_E_hist, g_ee_hist):
        H, tape = ctx.saved_tensors
        plan = ctx.plan
        if g_f_hist is not None and g_f_hist.numel() == 0:
            g_f_hist = None
        g_fiv, g_H = plan.backward(H, ctx.n_steps, tape if tape.numel() else None, ctx.every,
                                   g_f_final, g_f_hist, g_E_hist, g_ee_hist)
        # inputs that need no gradient get none (no cast launched for them)
        return (g_fiv.to(device=ctx.f_device, dtype=ctx.f_dtype) if ctx.needs_input_grad[0] else None,
                g_H.to(device=ctx.H_device, dtype=ctx.H_dtype) if ctx.needs_input_grad[1] else None,
                None, None, None)


def run_forward_jax_compatible(f_iv, H, t_final, solver_instance: WarpVlasovPoissonSolver):
    """Functional wrapper (solver.py:1413-1417), here over ``run_forward_torch``."""
    return solver_instance.run_forward_torch(f_iv, H, t_final)
