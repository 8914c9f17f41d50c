"""Host-side behaviour that needs no GPU: mesh construction, constructor validation with the
reference's messages, the ABI's exported symbols, and error reporting without a device."""

from __future__ import annotations

import ctypes
import os
import re

import numpy as np
import pytest
import torch

from conftest import ROOT
from warp_vp_solver_b200 import Mesh, WarpVlasovPoissonSolver, make_mesh
from warp_vp_solver_b200 import _capi


# --- mesh (reference tests/test_mesh.py) ------------------------------------------------------

def test_make_mesh_shapes(small_mesh):
    assert small_mesh.X.shape == (small_mesh.nx, small_mesh.nv)
    assert small_mesh.V.shape == (small_mesh.nx, small_mesh.nv)
    assert small_mesh.xs.shape == (small_mesh.nx,)
    assert small_mesh.vs.shape == (small_mesh.nv,)


def test_make_mesh_periodic_endpoints(small_mesh):
    assert small_mesh.xs[0] == 0.0
    np.testing.assert_allclose(small_mesh.xs[-1] + small_mesh.dx, small_mesh.period_x)
    np.testing.assert_allclose(small_mesh.vs[-1] + small_mesh.dv, small_mesh.period_v)


def test_make_mesh_dx_dv():
    mesh = make_mesh(length_x=2.0, length_v=3.0, nx=4, nv=6)
    np.testing.assert_allclose(mesh.dx, 0.5)
    np.testing.assert_allclose(mesh.dv, 1.0)


def test_meshgrid_consistency(small_mesh):
    np.testing.assert_array_equal(small_mesh.X[:, 0], small_mesh.xs)
    np.testing.assert_array_equal(small_mesh.V[0, :], small_mesh.vs)
    assert isinstance(make_mesh(1.0, 1.0, 8, 8), Mesh)


# --- constructor validation (reference solver.py:141-167, tests/test_optimized.py) ------------

def test_f_eq_shape_error(small_mesh):
    with pytest.raises(ValueError, match=r"f_eq shape \(4, 4\) != \(16, 32\)"):
        WarpVlasovPoissonSolver(small_mesh, 0.1, np.zeros((4, 4)))


def test_aggressive_requires_optimized(small_mesh):
    with pytest.raises(ValueError, match="aggressive=True requires optimized=True"):
        WarpVlasovPoissonSolver(small_mesh, 0.1, np.zeros((16, 32)), optimized=False,
                                aggressive=True)


def test_bad_layout_and_tile(small_mesh):
    with pytest.raises(ValueError, match="aggressive_layout must be one of"):
        WarpVlasovPoissonSolver(small_mesh, 0.1, np.zeros((16, 32)), aggressive_layout="x")
    with pytest.raises(ValueError, match="aggressive_tile_size must be positive"):
        WarpVlasovPoissonSolver(small_mesh, 0.1, np.zeros((16, 32)), aggressive_tile_size=0)


def test_legacy_rejects_record_history_false(small_mesh):
    s = WarpVlasovPoissonSolver(small_mesh, 0.001, np.zeros((16, 32)), optimized=False)
    with pytest.raises(ValueError, match="record_history=False"):
        s.run_forward(np.zeros((16, 32)), np.zeros(16), 5 * 0.001, record_history=False)


@pytest.mark.parametrize("layout", ["cpu_fused", "gpu_safe", "tiled"])
def test_aggressive_layouts_are_accepted(small_mesh, layout):
    s = WarpVlasovPoissonSolver(small_mesh, 0.001, np.zeros((16, 32)), aggressive=True,
                                aggressive_layout=layout)
    assert s.aggressive and s.aggressive_layout == layout


def test_num_steps_matches_python_int():
    m = make_mesh(10.0 * np.pi, 6.0, 8, 8)
    for dt, tf in ((0.05, 5.0), (0.05, 30.0), (0.001, 0.005), (0.1, 1.0), (0.9, 3.6)):
        s = WarpVlasovPoissonSolver(m, dt, np.zeros((8, 8)))
        assert s.num_steps(tf) == int(tf / dt)


# --- the C ABI ---------------------------------------------------------------------------------

def _header_functions():
    text = open(os.path.join(ROOT, "include", "vp_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vp_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _capi.load()
    declared = _header_functions()
    assert declared, "no functions parsed from include/vp_b200.h"
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in vp_b200.h but not exported"
    # every declared function has a ctypes signature in the binding
    missing = [n for n in declared if n not in _capi.SIGNATURES]
    assert not missing, f"no ctypes signature for {missing}"


def test_abi_version_and_error_reporting_without_device():
    lib = _capi.load()
    assert lib.vp_abi_version() == _capi.ABI_VERSION == 7
    assert lib.vp_plan_destroy(None) == 0
    out = ctypes.c_void_p()
    rc = lib.vp_plan_create(None, 0.1, None, 0, ctypes.byref(out))
    assert rc == _capi.VP_ERR_ARG
    assert "must not be NULL" in _capi.last_error()
    rc = lib.vp_forward(None, None, None, 1, None, None, None, None, None, 0, None, 0, None)
    assert rc == _capi.VP_ERR_ARG


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-device failure mode")
def test_plan_creation_fails_loudly_without_cuda(small_mesh):
    s = WarpVlasovPoissonSolver(small_mesh, 0.001, np.ones((16, 32)))
    with pytest.raises(RuntimeError, match="CUDA"):
        s.run_forward(np.ones((16, 32)), np.zeros(16), 0.005)


def test_non_finite_host_inputs_are_rejected_before_any_device_work(small_mesh):
    """NaN or infinite f_eq, f_iv or H given as host arrays raise ValueError on the host (the
    reference checks shapes only, solver.py:144-167)."""
    bad = np.ones((16, 32))
    bad[3, 4] = np.nan
    with pytest.raises(ValueError, match="f_eq contains NaN"):
        WarpVlasovPoissonSolver(small_mesh, 0.1, bad)
    s = WarpVlasovPoissonSolver(small_mesh, 0.1, np.ones((16, 32)))
    f = np.ones((16, 32))
    f[0, 0] = np.inf
    with pytest.raises(ValueError, match="f_iv contains NaN"):
        s.run_forward(f, np.zeros(16), 0.5)
    H = np.zeros(16)
    H[2] = -np.inf
    with pytest.raises(ValueError, match="H contains NaN"):
        s._run_backward(np.ones((16, 32)), H, 0.5, None, None, None, None, None)
    with pytest.raises(ValueError, match="H contains NaN"):
        s.run_forward_torch(np.ones((16, 32)), torch.tensor(H), 0.5)


def test_plan_create_rejects_non_finite_f_eq_in_the_c_abi(small_mesh):
    lib = _capi.load()
    xs = np.ascontiguousarray(small_mesh.xs, dtype=np.float64)
    vs = np.ascontiguousarray(small_mesh.vs, dtype=np.float64)
    desc = _capi.MeshDesc(16, 32, _capi.dbl_ptr(xs), _capi.dbl_ptr(vs), float(small_mesh.dx),
                          float(small_mesh.dv), float(small_mesh.period_x), float(small_mesh.period_v))
    f_eq = np.ones((16, 32))
    f_eq[5, 7] = np.nan
    out = ctypes.c_void_p()
    rc = lib.vp_plan_create(ctypes.byref(desc), 0.1, _capi.dbl_ptr(f_eq), _capi.VP_F32, ctypes.byref(out))
    assert rc == _capi.VP_ERR_ARG and out.value is None
    assert "f_eq[5, 7] is not finite" in _capi.last_error()
