"""Phase-space mesh, with the same fields and construction as the reference.

Mirrors ``warp_vp_solver/mesh.py:10-56``: x in [0, length_x) with ``nx`` points, v in
[-length_v, length_v) with ``nv`` points, both periodic, and ``V, X = meshgrid(vs, xs)`` so that
arrays are laid out (nx, nv) with x along rows. ``period_v`` is the half width ``length_v``;
the v period used by the advection is ``2 * period_v``.
"""

from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class Mesh:
    xs: np.ndarray
    dx: float
    vs: np.ndarray
    dv: float
    V: np.ndarray
    X: np.ndarray
    period_x: float
    period_v: float
    nx: int
    nv: int


def make_mesh(length_x: float, length_v: float, nx: int, nv: int) -> Mesh:
    """Build a periodic phase-space mesh (warp_vp_solver/mesh.py:26-56)."""
    xs = np.linspace(0.0, length_x, nx, endpoint=False, dtype=np.float64)
    dx = float(xs[1] - xs[0])
    vs = np.linspace(-length_v, length_v, nv, endpoint=False, dtype=np.float64)
    dv = float(vs[1] - vs[0])
    V, X = np.meshgrid(vs, xs)
    return Mesh(xs=xs, dx=dx, vs=vs, dv=dv, X=X, V=V, period_x=float(length_x),
                period_v=float(length_v), nx=int(nx), nv=int(nv))
