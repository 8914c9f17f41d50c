"""Spectral Poisson solve (reference: warp_vp_solver/poisson.py).

``fft_inv_multiplier`` is the host-side constant of the solve, computed exactly as the
reference does (poisson.py:34-45); the device plan rounds it to the compute type.
``solve_poisson`` / ``solve_poisson_adjoint`` run the hand-written in-block radix-2 FFT on the
device (the reference's host NumPy round trip, poisson.py:48-99, and its ``wp.tile_fft``
placeholder, poisson.py:108-179, are what this replaces).
"""

from __future__ import annotations

import numpy as np
import torch

from .mesh import make_mesh
from .plan import Plan


def fft_inv_multiplier(nx: int, period_x: float) -> np.ndarray:
    """Spectral multiplier -1/(i*k) with k = 2*pi*fftfreq; the k=0 entry is zero."""
    freqs = np.fft.fftfreq(nx, d=period_x / nx)
    mult = np.zeros(nx, dtype=np.complex128)
    nonzero = freqs != 0.0
    mult[nonzero] = -1.0 / (1j * 2.0 * np.pi * freqs[nonzero])
    return mult


_plans: dict[tuple, Plan] = {}


def _poisson_plan(nx: int, period_x: float, dtype, device) -> Plan:
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    key = (int(nx), float(period_x), str(dtype), str(dev))
    p = _plans.get(key)
    if p is None:
        mesh = make_mesh(period_x, 1.0, nx, 2)
        p = Plan(mesh, 1.0, np.zeros((nx, 2)), dtype=dtype, device=dev)
        _plans[key] = p
    return p


def solve_poisson(rho, period_x: float, *, dtype=torch.float32, device=None):
    """E = real(ifft(m * fft(rho))) on the device. NumPy in -> NumPy float64 out."""
    nx = int(np.shape(rho)[0])
    p = _poisson_plan(nx, period_x, dtype, device)
    E = p.poisson(rho, adjoint=False)
    return E if isinstance(rho, torch.Tensor) else E.double().cpu().numpy()


def solve_poisson_adjoint(g_E, period_x: float, *, dtype=torch.float32, device=None):
    """rho_bar = real(ifft(conj(m) * fft(g_E))) on the device (poisson.py:72-99)."""
    nx = int(np.shape(g_E)[0])
    p = _poisson_plan(nx, period_x, dtype, device)
    out = p.poisson(g_E, adjoint=True)
    return out if isinstance(g_E, torch.Tensor) else out.double().cpu().numpy()
