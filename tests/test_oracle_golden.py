"""The CPU oracle is pinned to golden vectors recorded from the reference's own code.

``tests/golden/make_golden.py`` ran the reference's ``warp_vp_solver`` kernels and solver
(legacy ``optimized=False`` path) under a serial Warp interpreter. The literal oracle must
reproduce every array bit for bit; the index-space delta-f oracle (the scheme the CUDA kernels
evaluate) must agree to float64 round-off.
"""

from __future__ import annotations

import os

import numpy as np
import pytest

import vp_oracle as O
from conftest import BACKWARD_CASES, FORWARD_CASES

FIELDS = ("f_final", "f_hist", "E_hist", "ee_hist")


@pytest.mark.parametrize("case", FORWARD_CASES, ids=lambda c: c.name)
def test_literal_forward_bit_exact(case):
    out = O.run_forward(case.grid, float(case["dt"]), case["f_eq"], case["f_iv"], case["H"],
                        float(case["t_final"]))
    for arr, name in zip(out, FIELDS):
        np.testing.assert_array_equal(arr, case[name], err_msg=f"{case.name}:{name}")


@pytest.mark.parametrize("case", FORWARD_CASES, ids=lambda c: c.name)
def test_delta_forward_matches_reference(case):
    T = int(case["n_steps"])
    out = O.delta_forward(case.grid, float(case["dt"]), case["f_eq"], case["f_iv"], case["H"], T)
    for arr, name in zip(out, FIELDS):
        ref = case[name]
        if case.name.startswith("fwd_equilibrium") and name in ("E_hist", "ee_hist"):
            # the reference's field is pure round-off (~1e-18); the delta form gives exactly 0
            assert np.abs(arr).max() <= 1e-15, f"{case.name}:{name}"
            continue
        # max-norm relative error: max|a - b| / max|b|
        assert O.rel_err(arr, ref) < 1e-11, f"{case.name}:{name}: {O.rel_err(arr, ref):.2e}"


@pytest.mark.parametrize("case", BACKWARD_CASES, ids=lambda c: c.name)
def test_literal_backward_bit_exact(case):
    g = case.grid
    dt, t_final = float(case["dt"]), float(case["t_final"])
    fwd = O.run_forward(g, dt, case["f_eq"], case["f_iv"], case["H"], t_final)
    np.testing.assert_array_equal(fwd[0], case["f_final"])
    g_f, g_H = O.run_backward(g, dt, case["f_eq"], case["f_iv"], case["H"], t_final, fwd[1],
                              case["g_f_final"], case["g_f_hist"], case["g_E_hist"],
                              case["g_ee_hist"])
    np.testing.assert_array_equal(g_f, case["g_f_iv"])
    np.testing.assert_array_equal(g_H, case["g_H"])


@pytest.mark.parametrize("case", BACKWARD_CASES, ids=lambda c: c.name)
def test_delta_backward_matches_reference(case):
    T = int(case["n_steps"])
    g_f, g_H = O.delta_backward(case.grid, float(case["dt"]), case["f_eq"], case["f_iv"],
                                case["H"], T, case["g_f_final"], case["g_f_hist"],
                                case["g_E_hist"], case["g_ee_hist"])
    assert O.rel_err(g_f, case["g_f_iv"]) < 1e-11
    assert O.rel_err(g_H, case["g_H"]) < 1e-11


def test_literal_kernels_bit_exact(golden_kernels):
    k = golden_kernels
    g = O.make_grid(float(k["mesh_length_x"]), float(k["mesh_length_v"]), int(k["mesh_nx"]),
                    int(k["mesh_nv"]))
    f_eq, f_iv = k["f_eq"], k["f_iv"]
    np.testing.assert_array_equal(O.semilag_x(f_iv, g, float(k["x_dt"])), k["x_out"])
    np.testing.assert_array_equal(O.semilag_v(f_iv, k["v_E"], g, float(k["v_dt"])), k["v_out"])
    np.testing.assert_array_equal(O.compute_rho(f_eq, f_iv, g.dv), k["rho"])
    assert O.compute_ee(k["ee_E"], g.dx) == k["ee"][0]
    np.testing.assert_array_equal(O.semilag_x_adjoint(k["xadj_g_out"], g, float(k["xadj_dt"])),
                                  k["xadj_g_in"])
    g_in, g_E = O.semilag_v_adjoint(k["vadj_g_out"], f_iv, k["vadj_E"], g, float(k["vadj_dt"]))
    np.testing.assert_array_equal(g_in, k["vadj_g_in"])
    np.testing.assert_array_equal(g_E, k["vadj_g_E"])
    np.testing.assert_array_equal(O.compute_rho_adjoint(k["rhoadj_g_rho"], g.nv, g.dv),
                                  k["rhoadj_g_f"])
    np.testing.assert_array_equal(O.compute_ee_adjoint(1.0, k["eeadj_E"], g.dx), k["eeadj_g_E"])
    mult = O.fft_inv_multiplier(g.nx, g.period_x)
    np.testing.assert_array_equal(mult.real, k["poisson_mult_re"])
    np.testing.assert_array_equal(mult.imag, k["poisson_mult_im"])
    np.testing.assert_array_equal(O.solve_poisson(k["poisson_rho"], g.period_x), k["poisson_E"])
    np.testing.assert_array_equal(O.solve_poisson_adjoint(k["poisson_g_E"], g.period_x),
                                  k["poisson_adj"])


def _c_oracle():
    import subprocess

    import vp_oracle_c as OC
    if not OC.available():
        subprocess.run(["make", "-C", os.path.join(os.path.dirname(__file__), "..", "oracle")],
                       check=True, capture_output=True)
    assert OC.available(), "oracle/_build/libvporacle.so did not build"
    return OC


@pytest.mark.parametrize("case", FORWARD_CASES, ids=lambda c: c.name)
def test_c_oracle_forward_matches_reference(case):
    """The OpenMP C restatement (the timed CPU baseline) reproduces the reference's outputs."""
    OC = _c_oracle()
    out = OC.forward(case.grid, float(case["dt"]), case["f_eq"], case["f_iv"], case["H"],
                     int(case["n_steps"]))
    for arr, name in zip(out, FIELDS):
        assert O.rel_err(arr, case[name]) < 1e-13, name


@pytest.mark.parametrize("case", BACKWARD_CASES, ids=lambda c: c.name)
def test_c_oracle_backward_matches_reference(case):
    OC = _c_oracle()
    T, dt = int(case["n_steps"]), float(case["dt"])
    fwd = OC.forward(case.grid, dt, case["f_eq"], case["f_iv"], case["H"], T)
    g_f, g_H = OC.backward(case.grid, dt, case["f_eq"], case["f_iv"], case["H"], T, fwd[1],
                           case["g_f_final"], case["g_f_hist"], case["g_E_hist"], case["g_ee_hist"])
    assert O.rel_err(g_f, case["g_f_iv"]) < 1e-13
    assert O.rel_err(g_H, case["g_H"]) < 1e-13



def _aggressive_cases():
    from conftest import load_golden
    return load_golden("aggressive")


@pytest.mark.parametrize("case", _aggressive_cases(), ids=lambda c: c.name)
def test_literal_aggressive_forward_and_backward_bit_exact(case):
    """The merged-Strang (aggressive) loops of the reference, solver.py:618-736 and 1111-1338,
    recorded for the cpu_fused and gpu_safe layouts."""
    g = case.grid
    dt, t_final = float(case["dt"]), float(case["t_final"])
    out = O.run_forward_aggressive(g, dt, case["f_eq"], case["f_iv"], case["H"], t_final)
    for arr, name in zip(out, FIELDS):
        np.testing.assert_array_equal(arr, case[name], err_msg=f"{case.name}:{name}")
    g_f, g_H = O.run_backward_aggressive(g, dt, case["f_eq"], case["f_iv"], case["H"], t_final,
                                         out[1], case["g_f_final"], case["g_f_hist"],
                                         case["g_E_hist"], case["g_ee_hist"])
    np.testing.assert_array_equal(g_f, case["g_f_iv"])
    np.testing.assert_array_equal(g_H, case["g_H"])
