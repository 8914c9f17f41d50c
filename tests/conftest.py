"""Shared fixtures. Tests marked ``gpu`` need a CUDA device and the built library; the rest
run on CPU (oracle vs golden vectors, host logic, ABI exports, multi-rank logic over gloo)."""

from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libvpb200.so")
    config.addinivalue_line("markers", "slow: long-running parity case")


class GoldenCase:
    """One named case of a golden .npz file (keys '<case>/<field>')."""

    def __init__(self, data, name):
        self.name = name
        self._d = data

    def __getitem__(self, k):
        return self._d[f"{self.name}/{k}"]

    def has(self, k):
        return f"{self.name}/{k}" in self._d

    @property
    def mesh(self):
        from warp_vp_solver_b200 import make_mesh
        return make_mesh(float(self["mesh_length_x"]), float(self["mesh_length_v"]),
                         int(self["mesh_nx"]), int(self["mesh_nv"]))

    @property
    def grid(self):
        import vp_oracle
        return vp_oracle.make_grid(float(self["mesh_length_x"]), float(self["mesh_length_v"]),
                                   int(self["mesh_nx"]), int(self["mesh_nv"]))


def load_golden(kind):
    data = np.load(os.path.join(GOLDEN, f"golden_{kind}.npz"))
    names = sorted({k.split("/")[0] for k in data.files})
    return [GoldenCase(data, n) for n in names]


FORWARD_CASES = load_golden("forward")
BACKWARD_CASES = load_golden("backward")


@pytest.fixture(scope="session")
def golden_kernels():
    return dict(np.load(os.path.join(GOLDEN, "golden_kernels.npz")))


def two_stream_state(mesh, mu=2.4, eps=1e-3, k=0.2):
    f_eq = (np.exp(-0.5 * (mesh.V - mu) ** 2) + np.exp(-0.5 * (mesh.V + mu) ** 2)) / (
        2.0 * np.sqrt(2.0 * np.pi))
    return f_eq, (1.0 + eps * np.cos(k * mesh.X)) * f_eq


@pytest.fixture
def small_mesh():
    from warp_vp_solver_b200 import make_mesh
    return make_mesh(length_x=2.0 * np.pi, length_v=6.0, nx=16, nv=32)


@pytest.fixture
def two_stream_mesh():
    from warp_vp_solver_b200 import make_mesh
    return make_mesh(length_x=10.0 * np.pi, length_v=6.0, nx=64, nv=64)


# Measured errors of the parity tests at the configurations' sizes, printed after the run (also
# under -q) so that a GPU run's log shows how far each bar is from what the kernels achieve.
MEASURED: list[tuple[str, float, float]] = []


@pytest.fixture
def record_error():
    def rec(name: str, err: float, bar: float) -> float:
        MEASURED.append((name, float(err), float(bar)))
        return float(err)
    return rec


def pytest_terminal_summary(terminalreporter):
    if not MEASURED:
        return
    terminalreporter.write_line("measured max-norm relative errors (value / bar):")
    for name, err, bar in MEASURED:
        terminalreporter.write_line(f"  {name:<46s} {err:9.2e} / {bar:7.1e}")
