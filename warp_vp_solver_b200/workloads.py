"""Synthetic problem set-ups of the benchmark configurations (seeded, no datasets).

* ``two_stream``: f_eq = [exp(-(v-mu)^2/2) + exp(-(v+mu)^2/2)] / (2 sqrt(2 pi)),
  f_iv = (1 + eps cos(k x)) f_eq (the reference's tests/conftest.py:28-37 and notebooks).
* ``bump_on_tail``: f_eq = 0.9/sqrt(2 pi) exp(-v^2/2) + 0.2/sqrt(2 pi)/0.5 exp(-(v-4.5)^2/(2*0.25)),
  f_iv = (1 + 0.04 cos(0.3 x)) f_eq.
* ``fourier_coefficients``: seeded (2, n_modes) coefficients a_k, b_k = std * N(0, 1) (the
  reference's tests draw ``scale * standard_normal``, so "N(0, s)" is read as standard deviation s)
  for H(x) = sum_k a_k cos(k0 k x) + b_k sin(k0 k x) with k0 = 2 pi / length_x.
"""

from __future__ import annotations

import dataclasses

import numpy as np

from .mesh import Mesh, make_mesh


def two_stream(mesh: Mesh, mu: float = 2.4, eps: float = 1e-3, k: float = 0.2):
    f_eq = (np.exp(-0.5 * (mesh.V - mu) ** 2) + np.exp(-0.5 * (mesh.V + mu) ** 2)) / (
        2.0 * np.sqrt(2.0 * np.pi))
    return f_eq, (1.0 + eps * np.cos(k * mesh.X)) * f_eq


def bump_on_tail(mesh: Mesh, eps: float = 0.04, k: float = 0.3):
    V = mesh.V
    f_eq = 0.9 / np.sqrt(2.0 * np.pi) * np.exp(-0.5 * V ** 2) + \
        0.2 / np.sqrt(2.0 * np.pi) / 0.5 * np.exp(-((V - 4.5) ** 2) / (2.0 * 0.25))
    return f_eq, (1.0 + eps * np.cos(k * mesh.X)) * f_eq


def fourier_coefficients(n_modes: int, std: float, seed: int) -> np.ndarray:
    return std * np.random.default_rng(seed).standard_normal((2, n_modes))


def fourier_field(coeffs: np.ndarray, xs: np.ndarray, k0: float) -> np.ndarray:
    n = coeffs.shape[1]
    k = np.arange(1, n + 1)
    return coeffs[0] @ np.cos(k0 * k[:, None] * xs) + coeffs[1] @ np.sin(k0 * k[:, None] * xs)


@dataclasses.dataclass
class Workload:
    name: str
    description: str
    mesh: Mesh
    dt: float
    t_final: float
    f_eq: np.ndarray
    f_iv: np.ndarray
    coeffs: np.ndarray | None
    k0: float
    adjoint: bool
    checkpoint_every: int | None

    @property
    def n_steps(self) -> int:
        return int(self.t_final / self.dt)

    @property
    def H(self) -> np.ndarray:
        if self.coeffs is None:
            return np.zeros(self.mesh.nx)
        return fourier_field(self.coeffs, self.mesh.xs, self.k0)


def make_workload(name: str) -> Workload:
    """The single-instance benchmark configurations by name: c1, c2, c3, c5 (one instance of the
    surrogate's training data), roofline."""
    if name == "c1":
        m = make_mesh(10.0 * np.pi, 6.0, 128, 128)
        f_eq, f_iv = two_stream(m)
        return Workload("c1", "two-stream 128x128, dt 0.05, 100 steps, H=0, forward", m, 0.05, 5.0,
                        f_eq, f_iv, None, 2 * np.pi / m.period_x, False, None)
    if name == "c2":
        m = make_mesh(10.0 * np.pi, 6.0, 256, 256)
        f_eq, f_iv = two_stream(m)
        return Workload("c2", "two-stream 256x256, dt 0.05, 100 steps, 8-mode H (std 1e-2, seed 0), "
                        "forward + adjoint of J = sum(ee)*dt", m, 0.05, 5.0, f_eq, f_iv,
                        fourier_coefficients(8, 1e-2, 0), 2 * np.pi / m.period_x, True, None)
    if name == "c3":
        lx = 2.0 * np.pi / 0.3
        m = make_mesh(lx, 8.0, 512, 1024)
        f_eq, f_iv = bump_on_tail(m)
        return Workload("c3", "bump-on-tail 512x1024, dt 0.05, 600 steps, 16-mode H (std 1e-2, seed 0), "
                        "sqrt(n)-checkpointed forward + adjoint of J = sum(ee)*dt", m, 0.05, 30.0,
                        f_eq, f_iv, fourier_coefficients(16, 1e-2, 0), 2 * np.pi / lx, True, 25)
    if name == "c5":
        m = make_mesh(10.0 * np.pi, 6.0, 256, 256)
        f_eq, f_iv = two_stream(m)
        return Workload("c5", "one surrogate training sample: two-stream 256x256, dt 0.05, 100 steps, "
                        "16-mode H (std 0.05, seed 0), forward", m, 0.05, 5.0, f_eq, f_iv,
                        fourier_coefficients(16, 0.05, 0), 2 * np.pi / m.period_x, False, None)
    if name == "roofline":
        m = make_mesh(10.0 * np.pi, 6.0, 8192, 8192)
        f_eq, f_iv = two_stream(m)
        return Workload("roofline", "two-stream 8192x8192 (268 MB of state, > L2), dt 0.05, 20 steps, "
                        "8-mode H, sqrt(n)-checkpointed forward + adjoint of J = sum(ee)*dt", m, 0.05,
                        1.0, f_eq, f_iv, fourier_coefficients(8, 1e-2, 0), 2 * np.pi / m.period_x,
                        True, None)
    raise ValueError(f"unknown workload {name!r}")


@dataclasses.dataclass
class EnsembleWorkload:
    """Independent instances sharing dt and the number of steps."""
    name: str
    description: str
    dt: float
    t_final: float
    meshes: list
    f_eqs: list
    f_ivs: list
    coeffs: list
    adjoint: bool = True

    @property
    def n(self) -> int:
        return len(self.meshes)

    @property
    def n_steps(self) -> int:
        return int(self.t_final / self.dt)

    @property
    def cells(self) -> int:
        return int(sum(m.nx * m.nv for m in self.meshes))

    def k0(self, i: int) -> float:
        return 2 * np.pi / self.meshes[i].period_x

    def H(self, i: int) -> np.ndarray:
        return fourier_field(self.coeffs[i], self.meshes[i].xs, self.k0(i))

    def subset(self, idx) -> "EnsembleWorkload":
        idx = list(idx)
        return EnsembleWorkload(self.name, self.description, self.dt, self.t_final,
                                [self.meshes[i] for i in idx], [self.f_eqs[i] for i in idx],
                                [self.f_ivs[i] for i in idx], [self.coeffs[i] for i in idx],
                                self.adjoint)


def make_ensemble_workload(name: str = "c4", n_instances: int = 256, seed: int = 0) -> EnsembleWorkload:
    """Uneven two-stream ensemble: nx ~ U{64,128,256}, nv ~ U{128,256,512}, mu ~ U[2,3],
    perturbation amplitude ~ U[1e-4,1e-2] on cos(0.2 x), L_x = 10 pi, v in [-6, 6), 8-mode H
    with coefficients of standard deviation 1e-2; dt 0.05, 100 steps, forward + adjoint."""
    if name != "c4":
        raise ValueError(f"unknown ensemble workload {name!r}")
    rng = np.random.default_rng(seed)
    meshes, f_eqs, f_ivs, coeffs = [], [], [], []
    cache: dict = {}
    for _ in range(n_instances):
        nx = int(rng.choice([64, 128, 256]))
        nv = int(rng.choice([128, 256, 512]))
        mu = float(rng.uniform(2.0, 3.0))
        eps = float(rng.uniform(1e-4, 1e-2))
        m = cache.setdefault((nx, nv), make_mesh(10.0 * np.pi, 6.0, nx, nv))
        f_eq, f_iv = two_stream(m, mu=mu, eps=eps)
        meshes.append(m)
        f_eqs.append(f_eq)
        f_ivs.append(f_iv)
        coeffs.append(1e-2 * rng.standard_normal((2, 8)))
    return EnsembleWorkload("c4", f"{n_instances} uneven two-stream instances, nx in {{64,128,256}}, "
                            "nv in {128,256,512}, dt 0.05, 100 steps, 8-mode H, forward + adjoint "
                            "of J = sum(ee)*dt per instance", 0.05, 5.0, meshes, f_eqs, f_ivs, coeffs)
