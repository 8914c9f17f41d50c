"""Generate golden vectors by running the reference's own code.

Run from the repository root, in a container where the reference checkout is
present::

    python tests/golden/make_golden.py [--ref /path/to/reference]

The reference (Forgotten/warp_vp_solver) is pure Python on top of NVIDIA
Warp and JAX, neither of which can be installed offline. This script puts
``tests/golden/_shims`` first on ``sys.path`` (a serial per-thread Warp
interpreter and an import-only JAX stub), imports the reference's
``warp_vp_solver.mesh`` / ``.kernels`` / ``.poisson`` / ``.solver`` modules
directly from the checkout (skipping its ``__init__``, which pulls in
matplotlib), and calls:

* ``WarpVlasovPoissonSolver(..., optimized=False).run_forward``
  (``warp_vp_solver/solver.py:418-524``),
* ``WarpVlasovPoissonSolver(..., optimized=False)._run_backward``
  (``warp_vp_solver/solver.py:742-932``),
* the single-stage kernels of ``warp_vp_solver/kernels.py:109-322`` through
  ``wp.launch`` exactly as ``tests/test_kernels.py`` launches them,
* ``warp_vp_solver/poisson.py:34-99``,
* ``WarpVlasovPoissonSolver(..., optimized=True, aggressive=True)`` forward and
  ``_run_backward`` (``warp_vp_solver/solver.py:618-736, 1111-1338``).

The outputs are written to ``tests/golden/golden_*.npz`` (float64). The cases
mirror the reference's own test fixtures (``tests/conftest.py``,
``tests/test_solver.py``, ``tests/test_optimized.py``,
``tests/test_kernels.py``) plus a few edge cases of the same API (an
x-dependent equilibrium, large semi-Lagrangian shifts, a non-power-of-two
grid, every cotangent non-zero).
"""

from __future__ import annotations

import argparse
import importlib
import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load_reference(ref_root: str):
    sys.path.insert(0, os.path.join(HERE, "_shims"))
    pkg = types.ModuleType("warp_vp_solver")
    pkg.__path__ = [os.path.join(ref_root, "warp_vp_solver")]
    sys.modules["warp_vp_solver"] = pkg
    mods = types.SimpleNamespace()
    mods.mesh = importlib.import_module("warp_vp_solver.mesh")
    mods.kernels = importlib.import_module("warp_vp_solver.kernels")
    mods.poisson = importlib.import_module("warp_vp_solver.poisson")
    mods.solver = importlib.import_module("warp_vp_solver.solver")
    mods.wp = importlib.import_module("warp")
    return mods


# ---------------------------------------------------------------------------
# Problem set-ups (same formulas as the reference's fixtures)
# ---------------------------------------------------------------------------


def maxwell(mesh):
    # tests/test_solver.py:28-43
    f_eq = np.exp(-0.5 * mesh.V ** 2)
    f0 = f_eq * (1.0 + 0.001 * np.cos(mesh.X))
    return f_eq, f0


def two_stream(mesh, mu=2.4, eps=1e-3, k=0.2):
    # tests/conftest.py:28-37
    f_eq = (np.exp(-0.5 * (mesh.V - mu) ** 2) + np.exp(-0.5 * (mesh.V + mu) ** 2)) / (
        2.0 * np.sqrt(2.0 * np.pi)
    )
    f_iv = (1.0 + eps * np.cos(k * mesh.X)) * f_eq
    return f_eq, f_iv


def fourier_field(coeffs, xs, k0):
    # warp_vp_solver/utils.py:37-48 (NumPy form of external_electric_field)
    n = coeffs.shape[1]
    k = np.arange(1, n + 1)
    return coeffs[0, :] @ np.cos(k0 * k[:, None] * xs) + coeffs[1, :] @ np.sin(
        k0 * k[:, None] * xs
    )


def forward_cases(ref):
    mk = ref.mesh.make_mesh
    cases = []

    m = mk(2.0 * np.pi, 6.0, 16, 32)
    f_eq, f0 = maxwell(m)
    cases.append(("fwd_maxwell_16x32", m, f_eq, f0, np.zeros(m.nx), 0.001, 5 * 0.001))

    rng = np.random.default_rng(7)
    H = 0.01 * rng.standard_normal(m.nx)
    cases.append(("fwd_maxwell_H_16x32", m, f_eq, f0, H, 0.05, 10 * 0.05))

    m2 = mk(10.0 * np.pi, 6.0, 32, 32)
    f_eq2, f02 = two_stream(m2)
    cases.append(("fwd_twostream_32x32", m2, f_eq2, f02, np.zeros(m2.nx), 0.1, 1.0))

    # x-dependent equilibrium (the reference accepts any (nx, nv) f_eq)
    f_eq3 = np.exp(-0.5 * m.V ** 2) * (1.0 + 0.2 * np.cos(m.X))
    f03 = f_eq3 * (1.0 + 0.003 * np.sin(2.0 * m.X))
    H3 = 0.02 * np.random.default_rng(11).standard_normal(m.nx)
    cases.append(("fwd_feq2d_16x32", m, f_eq3, f03, H3, 0.05, 6 * 0.05))

    # large shifts: x half-step of several cells, v step of several cells
    H4 = 2.0 * np.random.default_rng(12).standard_normal(m.nx)
    cases.append(("fwd_bigshift_16x32", m, f_eq, f0, H4, 0.9, 4 * 0.9))

    # non-power-of-two grid
    m5 = mk(10.0 * np.pi, 6.0, 24, 40)
    f_eq5, f05 = two_stream(m5, eps=1e-2)
    H5 = fourier_field(0.05 * np.random.default_rng(13).standard_normal((2, 3)), m5.xs, 0.2)
    cases.append(("fwd_odd_24x40", m5, f_eq5, f05, H5, 0.1, 6 * 0.1))

    # equilibrium is a fixed point (tests/test_aggressive.py:295-304 applied to the plain path)
    cases.append(("fwd_equilibrium_16x32", m, f_eq, f_eq.copy(), np.zeros(m.nx), 0.05, 5 * 0.05))
    return cases


def backward_cases(ref):
    mk = ref.mesh.make_mesh
    cases = []

    # tests/test_optimized.py:217-248: cost = sum(f_final^2) + sum(E_hist^2) + sum(ee_hist)
    m = mk(2.0 * np.pi, 6.0, 16, 32)
    f_eq, f0 = maxwell(m)
    rng = np.random.default_rng(2)
    H = 0.001 * rng.standard_normal(m.nx)
    cases.append(("bwd_mix_16x32", m, f_eq, f0, H, 0.001, 5 * 0.001, "mix"))

    # time-integrated electric energy J = trapezoid(ee, dx=dt) (utils.py:111-116), 8-mode H
    m2 = mk(10.0 * np.pi, 6.0, 32, 32)
    f_eq2, f02 = two_stream(m2)
    coeffs = np.sqrt(1e-2) * np.random.default_rng(0).standard_normal((2, 8))
    H2 = fourier_field(coeffs, m2.xs, 2.0 * np.pi / (10.0 * np.pi))
    cases.append(("bwd_eet_twostream_32x32", m2, f_eq2, f02, H2, 0.05, 10 * 0.05, "eet"))

    # every cotangent random, including the f history
    H3 = 0.01 * np.random.default_rng(21).standard_normal(m.nx)
    cases.append(("bwd_random_16x32", m, f_eq, f0, H3, 0.05, 4 * 0.05, "random"))

    f_eq4 = np.exp(-0.5 * m.V ** 2) * (1.0 + 0.2 * np.cos(m.X))
    f04 = f_eq4 * (1.0 + 0.003 * np.sin(2.0 * m.X))
    cases.append(("bwd_feq2d_16x32", m, f_eq4, f04, H3, 0.05, 4 * 0.05, "random"))

    H5 = 2.0 * np.random.default_rng(12).standard_normal(m.nx)
    cases.append(("bwd_bigshift_16x32", m, f_eq, f0, H5, 0.9, 3 * 0.9, "random"))

    m6 = mk(10.0 * np.pi, 6.0, 24, 40)
    f_eq6, f06 = two_stream(m6, eps=1e-2)
    H6 = 0.05 * np.random.default_rng(14).standard_normal(m6.nx)
    cases.append(("bwd_odd_24x40", m6, f_eq6, f06, H6, 0.1, 4 * 0.1, "random"))
    return cases


def aggressive_cases(ref):
    """The merged-Strang (aggressive) path, solver.py:618-736 and 1111-1338."""
    mk = ref.mesh.make_mesh
    m = mk(2.0 * np.pi, 6.0, 16, 32)
    f_eq, f0 = maxwell(m)
    m2 = mk(10.0 * np.pi, 6.0, 32, 32)
    f_eq2, f02 = two_stream(m2, eps=1e-2)
    f_eq3 = np.exp(-0.5 * m.V ** 2) * (1.0 + 0.2 * np.cos(m.X))
    f03 = f_eq3 * (1.0 + 0.003 * np.sin(2.0 * m.X))
    m5 = mk(10.0 * np.pi, 6.0, 24, 40)
    f_eq5, f05 = two_stream(m5, eps=1e-2)
    return [
        ("agg_twostream_32x32", m2, f_eq2, f02, 0.02 * np.random.default_rng(31).standard_normal(m2.nx),
         0.1, 8 * 0.1, "cpu_fused"),
        ("agg_maxwell_H_16x32", m, f_eq, f0, 0.01 * np.random.default_rng(32).standard_normal(m.nx),
         0.05, 6 * 0.05, "gpu_safe"),
        ("agg_feq2d_16x32", m, f_eq3, f03, 0.02 * np.random.default_rng(33).standard_normal(m.nx),
         0.05, 5 * 0.05, "cpu_fused"),
        ("agg_bigshift_16x32", m, f_eq, f0, 2.0 * np.random.default_rng(34).standard_normal(m.nx),
         0.9, 3 * 0.9, "cpu_fused"),
        ("agg_odd_24x40", m5, f_eq5, f05, 0.05 * np.random.default_rng(35).standard_normal(m5.nx),
         0.1, 4 * 0.1, "gpu_safe"),
        ("agg_single_16x32", m, f_eq, f0, 0.01 * np.random.default_rng(36).standard_normal(m.nx),
         0.05, 1 * 0.05, "cpu_fused"),
    ]


def cotangents(kind, outs, nx, nv, T, dt, seed):
    f_final, f_hist, E_hist, ee_hist = outs
    if kind == "mix":
        return 2.0 * f_final, np.zeros((T, nx, nv)), 2.0 * E_hist, np.ones(T)
    if kind == "eet":
        w = np.full(T, dt)
        w[0] *= 0.5
        w[-1] *= 0.5
        return np.zeros((nx, nv)), np.zeros((T, nx, nv)), np.zeros((T, nx)), w
    rng = np.random.default_rng(seed)
    return (
        rng.standard_normal((nx, nv)),
        0.1 * rng.standard_normal((T, nx, nv)),
        rng.standard_normal((T, nx)),
        rng.standard_normal(T),
    )


def mesh_dict(m):
    return dict(
        length_x=m.period_x, length_v=m.period_v, nx=m.nx, nv=m.nv,
        xs=m.xs, vs=m.vs, dx=m.dx, dv=m.dv,
    )


def kernel_case(ref):
    """Single-stage kernels on the two-stream 64x64 state (tests/test_kernels.py)."""
    wp, K, P = ref.wp, ref.kernels, ref.poisson
    mesh = ref.mesh.make_mesh(10.0 * np.pi, 6.0, 64, 64)
    f_eq, f_iv = two_stream(mesh)
    nx, nv = mesh.nx, mesh.nv
    xs, vs = wp.array(mesh.xs, dtype=wp.float64), wp.array(mesh.vs, dtype=wp.float64)
    out = dict(f_eq=f_eq, f_iv=f_iv, **{"mesh_" + k: v for k, v in mesh_dict(mesh).items()})

    def launch_x(f, dt):
        b = wp.zeros((nx, nv), dtype=wp.float64)
        wp.launch(K.semilag_x_kernel, dim=(nx, nv), inputs=[
            wp.array(f, dtype=wp.float64), b, xs, vs, wp.float64(dt),
            wp.float64(mesh.dx), wp.int32(nx), wp.float64(mesh.period_x)])
        return b.numpy()

    def launch_v(f, E, dt):
        b = wp.zeros((nx, nv), dtype=wp.float64)
        wp.launch(K.semilag_v_kernel, dim=(nx, nv), inputs=[
            wp.array(f, dtype=wp.float64), b, vs, wp.array(E, dtype=wp.float64),
            wp.float64(dt), wp.float64(mesh.dv), wp.int32(nv), wp.float64(2.0 * mesh.period_v)])
        return b.numpy()

    out["x_dt"] = 0.1
    out["x_out"] = launch_x(f_iv, 0.1)
    rng = np.random.default_rng(0)
    E = 0.01 * rng.standard_normal(nx)
    out["v_E"], out["v_dt"], out["v_out"] = E, 0.05, launch_v(f_iv, E, 0.05)

    rho = wp.zeros(nx, dtype=wp.float64)
    wp.launch(K.compute_rho_kernel, dim=nx, inputs=[
        wp.array(f_eq, dtype=wp.float64), wp.array(f_iv, dtype=wp.float64), rho,
        wp.float64(mesh.dv), wp.int32(nv)])
    out["rho"] = rho.numpy()

    E1 = np.random.default_rng(1).standard_normal(nx)
    ee = wp.zeros(1, dtype=wp.float64)
    wp.launch(K.compute_ee_kernel, dim=1, inputs=[
        wp.array(E1, dtype=wp.float64), ee, wp.float64(mesh.dx), wp.int32(nx)])
    out["ee_E"], out["ee"] = E1, ee.numpy()

    g_out = np.random.default_rng(3).standard_normal((nx, nv))
    g_in = wp.zeros((nx, nv), dtype=wp.float64)
    wp.launch(K.semilag_x_adjoint_kernel, dim=(nx, nv), inputs=[
        wp.array(g_out, dtype=wp.float64), g_in, xs, vs, wp.float64(0.07),
        wp.float64(mesh.dx), wp.int32(nx), wp.float64(mesh.period_x)])
    out["xadj_g_out"], out["xadj_dt"], out["xadj_g_in"] = g_out, 0.07, g_in.numpy()

    rng4 = np.random.default_rng(4)
    g_out_v = rng4.standard_normal((nx, nv))
    E_v = 0.01 * rng4.standard_normal(nx)
    g_in_v = wp.zeros((nx, nv), dtype=wp.float64)
    g_E_v = wp.zeros(nx, dtype=wp.float64)
    wp.launch(K.semilag_v_adjoint_kernel, dim=(nx, nv), inputs=[
        wp.array(g_out_v, dtype=wp.float64), g_in_v, g_E_v, wp.array(f_iv, dtype=wp.float64),
        vs, wp.array(E_v, dtype=wp.float64), wp.float64(0.05), wp.float64(mesh.dv),
        wp.int32(nv), wp.float64(2.0 * mesh.period_v)])
    out.update(vadj_g_out=g_out_v, vadj_E=E_v, vadj_dt=0.05,
               vadj_g_in=g_in_v.numpy(), vadj_g_E=g_E_v.numpy())

    g_rho = np.random.default_rng(6).standard_normal(nx)
    g_f = wp.zeros((nx, nv), dtype=wp.float64)
    wp.launch(K.compute_rho_adjoint_kernel, dim=(nx, nv), inputs=[
        wp.array(g_rho, dtype=wp.float64), g_f, wp.float64(mesh.dv), wp.int32(nv)])
    out["rhoadj_g_rho"], out["rhoadj_g_f"] = g_rho, g_f.numpy()

    E7 = np.random.default_rng(7).standard_normal(nx)
    g_E7 = wp.zeros(nx, dtype=wp.float64)
    wp.launch(K.compute_ee_adjoint_kernel, dim=nx, inputs=[
        wp.array(np.array([1.0]), dtype=wp.float64), wp.array(E7, dtype=wp.float64), g_E7,
        wp.float64(mesh.dx), wp.int32(nx)])
    out["eeadj_E"], out["eeadj_g_E"] = E7, g_E7.numpy()

    # Poisson (poisson.py:34-99) on the same mesh and on tests/test_poisson.py's inputs
    rho_p = np.random.default_rng(8).standard_normal(nx)
    out["poisson_rho"] = rho_p
    out["poisson_mult_re"] = P.fft_inv_multiplier(nx, mesh.period_x).real
    out["poisson_mult_im"] = P.fft_inv_multiplier(nx, mesh.period_x).imag
    out["poisson_E"] = P.solve_poisson_host(rho_p, mesh.period_x)
    g_E_p = np.random.default_rng(9).standard_normal(nx)
    out["poisson_g_E"] = g_E_p
    out["poisson_adj"] = P.solve_poisson_host_adjoint(g_E_p, mesh.period_x)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ap.add_argument("--out", default=HERE)
    args = ap.parse_args()
    ref = load_reference(args.ref)
    Solver = ref.solver.WarpVlasovPoissonSolver

    t0 = time.time()
    fwd = {}
    for name, m, f_eq, f_iv, H, dt, t_final in forward_cases(ref):
        s = Solver(mesh=m, dt=dt, f_eq=f_eq, optimized=False)
        f_final, f_hist, E_hist, ee_hist = s.run_forward(f_iv, H, t_final)
        T = s.num_steps(t_final)
        d = dict(f_eq=f_eq, f_iv=f_iv, H=H, dt=dt, t_final=t_final, n_steps=T,
                 f_final=f_final, f_hist=f_hist, E_hist=E_hist, ee_hist=ee_hist,
                 **{"mesh_" + k: v for k, v in mesh_dict(m).items()})
        for k, v in d.items():
            fwd[f"{name}/{k}"] = np.asarray(v)
        print(f"{name}: T={T} ({time.time() - t0:.1f}s)")
    np.savez_compressed(os.path.join(args.out, "golden_forward.npz"), **fwd)

    bwd = {}
    for i, (name, m, f_eq, f_iv, H, dt, t_final, kind) in enumerate(backward_cases(ref)):
        s = Solver(mesh=m, dt=dt, f_eq=f_eq, optimized=False)
        outs = s.run_forward(f_iv, H, t_final)
        T = s.num_steps(t_final)
        g_ff, g_fh, g_Eh, g_ee = cotangents(kind, outs, m.nx, m.nv, T, dt, 100 + i)
        g_f_iv, g_H = s._run_backward(f_iv, H, t_final, outs[1], g_ff, g_fh, g_Eh, g_ee)
        d = dict(f_eq=f_eq, f_iv=f_iv, H=H, dt=dt, t_final=t_final, n_steps=T,
                 f_final=outs[0], E_hist=outs[2], ee_hist=outs[3],
                 g_f_final=g_ff, g_f_hist=g_fh, g_E_hist=g_Eh, g_ee_hist=g_ee,
                 g_f_iv=g_f_iv, g_H=g_H,
                 **{"mesh_" + k: v for k, v in mesh_dict(m).items()})
        for k, v in d.items():
            bwd[f"{name}/{k}"] = np.asarray(v)
        print(f"{name}: T={T} ({time.time() - t0:.1f}s)")
    np.savez_compressed(os.path.join(args.out, "golden_backward.npz"), **bwd)

    kern = kernel_case(ref)
    np.savez_compressed(os.path.join(args.out, "golden_kernels.npz"), **kern)
    print(f"kernels ({time.time() - t0:.1f}s)")

    agg = {}
    for i, (name, m, f_eq, f_iv, H, dt, t_final, layout) in enumerate(aggressive_cases(ref)):
        s = Solver(mesh=m, dt=dt, f_eq=f_eq, optimized=True, aggressive=True, aggressive_layout=layout)
        outs = s.run_forward(f_iv, H, t_final)
        T = s.num_steps(t_final)
        g_ff, g_fh, g_Eh, g_ee = cotangents("random", outs, m.nx, m.nv, T, dt, 200 + i)
        g_f_iv, g_H = s._run_backward(f_iv, H, t_final, outs[1], g_ff, g_fh, g_Eh, g_ee)
        d = dict(f_eq=f_eq, f_iv=f_iv, H=H, dt=dt, t_final=t_final, n_steps=T,
                 f_final=outs[0], f_hist=outs[1], E_hist=outs[2], ee_hist=outs[3],
                 g_f_final=g_ff, g_f_hist=g_fh, g_E_hist=g_Eh, g_ee_hist=g_ee,
                 g_f_iv=g_f_iv, g_H=g_H, layout=layout,
                 **{"mesh_" + k: v for k, v in mesh_dict(m).items()})
        for k, v in d.items():
            agg[f"{name}/{k}"] = np.asarray(v)
        print(f"{name}: T={T} ({time.time() - t0:.1f}s)")
    np.savez_compressed(os.path.join(args.out, "golden_aggressive.npz"), **agg)


if __name__ == "__main__":
    main()
