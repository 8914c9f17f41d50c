"""Control parametrisation and cost functions in torch (reference: warp_vp_solver/utils.py).

The reference builds these on JAX so that ``jax.grad``/``optax`` can drive the optimisation;
here they are torch expressions around ``solver.run_forward_torch`` so that
``torch.autograd`` drives it. Plotting (utils.py:135-310) is not part of this package.
"""

from __future__ import annotations

from typing import Callable

import numpy as np
import torch


def _as_tensor(a, like: torch.Tensor | None = None) -> torch.Tensor:
    if isinstance(a, torch.Tensor):
        return a
    dtype = like.dtype if like is not None else torch.float64
    device = like.device if like is not None else None
    return torch.as_tensor(np.asarray(a), dtype=dtype, device=device)


_BASIS_CACHE: dict = {}


def _fourier_basis(xs: np.ndarray, N: int, k_0: float, dtype, device):
    """The stacked basis [cos(k0 k x); sin(k0 k x)] for k = 1..N on the mesh points, shape (2N, nx),
    built once per mesh, mode count, dtype and device (a host-to-device copy of the points inside
    every call would serialise the caller's stream with the host)."""
    key = (xs.tobytes(), int(N), float(k_0), dtype, str(device))
    hit = _BASIS_CACHE.get(key)
    if hit is None:
        k = torch.arange(1, N + 1, dtype=dtype, device=device)
        x = torch.as_tensor(xs, dtype=dtype, device=device)
        arg = k_0 * k[:, None] * x[None, :]
        hit = torch.cat([torch.cos(arg), torch.sin(arg)], dim=0).contiguous()
        if len(_BASIS_CACHE) >= 32:
            _BASIS_CACHE.clear()
        _BASIS_CACHE[key] = hit
    return hit


def external_electric_field(ak, mesh, k_0: float) -> torch.Tensor:
    """H(x) = sum_k a_k cos(k0 k x) + b_k sin(k0 k x) (utils.py:37-48). ``ak`` has shape (2, N).
    Evaluated as one product of the flattened coefficients with the stacked basis (one launch
    forward and one backward on the device)."""
    ak = _as_tensor(ak)
    N = ak.shape[1]
    basis = _fourier_basis(np.ascontiguousarray(mesh.xs, dtype=np.float64), N, k_0, ak.dtype, ak.device)
    return ak.reshape(2 * N) @ basis


def electric_energy_in_time(ee_array, solver) -> torch.Tensor:
    """Time-integrated electric energy trapezoid(ee, dx=dt) (utils.py:111-116)."""
    return torch.trapezoid(_as_tensor(ee_array), dx=solver.dt)


def _rel_entr(x: torch.Tensor, y: torch.Tensor) -> torch.Tensor:
    # scipy.special.rel_entr: x*log(x/y) for x>0, y>0; 0 for x==0, y>=0; inf otherwise
    pos = (x > 0) & (y > 0)
    safe_x = torch.where(pos, x, torch.ones_like(x))
    safe_y = torch.where(pos, y, torch.ones_like(y))
    val = torch.where(pos, safe_x * torch.log(safe_x / safe_y), torch.zeros_like(x))
    val = torch.where((x == 0) & (y >= 0), torch.zeros_like(x), val)
    bad = ~pos & ~((x == 0) & (y >= 0))
    return torch.where(bad, torch.full_like(x, float("inf")), val)


class _KLFunction(torch.autograd.Function):
    """KL(f || f_eq) and its gradient from the fused device kernels (vp_kl_divergence)."""

    @staticmethod
    def forward(ctx, f, plan, eps):
        value, grad = plan.kl_divergence(f.detach(), eps, want_grad=f.requires_grad)
        ctx.save_for_backward(grad if grad is not None else torch.empty(0, device=f.device))
        ctx.f_dtype = f.dtype
        return value.to(f.dtype)

    @staticmethod
    def backward(ctx, g):
        (grad,) = ctx.saved_tensors
        return (grad * g.to(grad.dtype)).to(ctx.f_dtype), None, None


def kl_divergence(f_T, solver, eps: float = 1e-12) -> torch.Tensor:
    """KL(f_T || f_eq) integrated over phase space (utils.py:53-76). A CUDA tensor goes through
    the fused device kernels of the solver's plan (value and gradient in one pass, float64);
    other inputs are evaluated with the same expression in torch."""
    if isinstance(f_T, torch.Tensor) and f_T.is_cuda and hasattr(solver, "plan"):
        return _KLFunction.apply(f_T, solver.plan, float(eps))
    f_T = _as_tensor(f_T)
    xs = torch.as_tensor(solver.mesh.xs, dtype=f_T.dtype, device=f_T.device)
    vs = torch.as_tensor(solver.mesh.vs, dtype=f_T.dtype, device=f_T.device)
    f_eq = torch.as_tensor(solver.f_eq, dtype=f_T.dtype, device=f_T.device)
    norm_final = torch.trapezoid(torch.trapezoid(f_T, vs, dim=1), xs) + eps
    norm_eq = torch.trapezoid(torch.trapezoid(f_eq, vs, dim=1), xs) + eps
    return torch.trapezoid(
        torch.trapezoid(_rel_entr(f_T / norm_final, f_eq / norm_eq + eps), vs, dim=1), xs)


def make_cost_function_kl(solver, solver_jit: Callable, f_iv, k_0: float,
                          t_final: float) -> Callable:
    """KL-divergence cost of the external-field coefficients (utils.py:79-92)."""
    def cost_function_kl(a_k):
        H = external_electric_field(a_k, solver.mesh, k_0)
        f_array, _, _, _ = solver_jit(f_iv, H, t_final)
        return kl_divergence(f_array, solver)
    return cost_function_kl


def make_cost_function_ee(solver, solver_jit: Callable, f_iv, k_0: float,
                          t_final: float) -> Callable:
    """Final-time electric energy cost (utils.py:95-108)."""
    def cost_function_ee(a_k):
        H = external_electric_field(a_k, solver.mesh, k_0)
        _, _, _, ee_array = solver_jit(f_iv, H, t_final)
        return ee_array[-1]
    return cost_function_ee


def make_cost_function_eet(solver, solver_jit: Callable, f_iv, k_0: float,
                           t_final: float) -> Callable:
    """Time-integrated electric energy cost (utils.py:119-132)."""
    def cost_function_eet(a_k):
        H = external_electric_field(a_k, solver.mesh, k_0)
        _, _, _, ee_array = solver_jit(f_iv, H, t_final)
        return electric_energy_in_time(ee_array, solver)
    return cost_function_eet
