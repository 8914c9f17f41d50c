"""Learned surrogate of the control-to-energy map, and surrogate-warm-started control.

The control is the external field H(x) = sum_k a_k cos(k0 k x) + b_k sin(k0 k x) of the
reference's ``external_electric_field`` (warp_vp_solver/utils.py:37-48); the cost is its
time-integrated electric energy J = trapezoid(ee, dt) (``make_cost_function_eet``,
utils.py:119-132), whose gradient the reference takes through its adjoint and optimises with
Adam from a random initial control (notebooks/01_Two_Stream_Warp.ipynb, cell 12).

* :func:`generate_dataset` runs many instances through the ensemble solver (one persistent launch
  per step for all of them) and records log ee at every step for random coefficient vectors.
* :class:`Surrogate` is the tensor-core MLP (``mlp.MLP``) on standardised inputs and outputs,
  trained by the project's own forward, backward and Adam kernels.
* :class:`ControlProblem` gives the true J and dJ/d(coefficients) through the fused forward and
  adjoint kernels; :func:`optimize_plain` is Adam on it until J stops improving;
  :func:`optimize_warm` first minimises the surrogate's J (:class:`SurrogateSearch`, one
  single-CTA launch running Adam through the network's forward and input gradient), then refines
  with the true gradient until J is within a tolerance of a target.
"""

from __future__ import annotations

import dataclasses
import time

import numpy as np
import torch

from .ensemble import Ensemble
from .mlp import MLP
from .plan import Plan


def fourier_basis(xs, k0: float, n_modes: int) -> np.ndarray:
    """(nx, 2 n_modes) matrix B with H = B @ concat(a, b)."""
    k = np.arange(1, n_modes + 1)
    arg = k0 * k[None, :] * np.asarray(xs)[:, None]
    return np.concatenate([np.cos(arg), np.sin(arg)], axis=1)


def trapezoid_weights(n: int, dt: float) -> np.ndarray:
    """w with sum(w * y) == trapezoid(y, dx=dt) for n samples."""
    w = np.full(n, float(dt))
    if n >= 2:
        w[0] = w[-1] = 0.5 * dt
    elif n == 1:
        w[0] = 0.0
    return w


@dataclasses.dataclass
class ControlSetup:
    mesh: object
    dt: float
    n_steps: int
    f_eq: np.ndarray
    f_iv: np.ndarray
    n_modes: int

    @property
    def k0(self) -> float:
        return 2.0 * np.pi / self.mesh.period_x

    @property
    def n_inputs(self) -> int:
        return 2 * self.n_modes


def generate_dataset(setup: ControlSetup, n_samples: int, coeff_std: float, seed: int,
                     chunk: int = 1024, dtype=torch.float32):
    """Random coefficient vectors (standard deviation ``coeff_std``) and the solver's log ee
    histories, (n, 2 n_modes) and (n, n_steps) float32 device tensors, plus timing."""
    rng = np.random.default_rng(seed)
    C = (coeff_std * rng.standard_normal((n_samples, setup.n_inputs))).astype(np.float32)
    dev = torch.device("cuda", torch.cuda.current_device())
    B = torch.tensor(fourier_basis(setup.mesh.xs, setup.k0, setup.n_modes), dtype=dtype, device=dev)
    Ct = torch.tensor(C, device=dev)
    out = torch.empty((n_samples, setup.n_steps), dtype=torch.float32, device=dev)
    chunk = min(chunk, n_samples)
    ens = Ensemble([setup.mesh] * chunk, setup.dt, [setup.f_eq] * chunk, dtype=dtype, device=dev)
    f_one = torch.tensor(np.asarray(setup.f_iv).reshape(-1), dtype=torch.float64, device=dev)
    f_iv = f_one.repeat(chunk)
    T = setup.n_steps
    bufs = ens.alloc_outputs(T, want_tape=False, want_f_final=False)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for s in range(0, n_samples, chunk):
        n = min(chunk, n_samples - s)
        H = Ct[s:s + n].to(dtype) @ B.T
        if n < chunk:
            H = torch.cat([H, torch.zeros((chunk - n, B.shape[0]), dtype=dtype, device=dev)])
        ens.forward_into(f_iv, H.reshape(-1).contiguous(), T, bufs)
        ee = bufs["ee_hist"].view(chunk, T)[:n]
        out[s:s + n] = torch.log(ee.float())
    torch.cuda.synchronize(dev)
    elapsed = time.perf_counter() - t0
    cell_steps = n_samples * setup.mesh.nx * setup.mesh.nv * T
    return Ct, out, {"seconds": elapsed, "cell_steps_per_s": cell_steps / elapsed,
                     "instances": n_samples, "chunk": chunk}


class Surrogate:
    """coefficients -> log ee history, an MLP on standardised inputs and outputs."""

    def __init__(self, n_inputs: int, n_outputs: int, hidden=(256, 256), max_batch: int = 4096,
                 seed: int = 0):
        self.widths = [n_inputs, *hidden, n_outputs]
        self.net = MLP(self.widths, max_batch=max_batch, seed=seed)
        self.x_scale = 1.0
        self.y_mean = None
        self.y_std = None

    def fit(self, X: torch.Tensor, Y: torch.Tensor, steps: int = 2000, batch: int = 1024,
            lr: float = 1e-3, seed: int = 0):
        """Adam on the mean-squared error of the standardised log ee; returns (loss history,
        seconds)."""
        self.x_scale = float(1.0 / X.float().std().item())
        self.y_mean = Y.float().mean(0)
        self.y_std = Y.float().std(0).clamp_min(1e-6)
        Xn = (X.float() * self.x_scale).contiguous()
        Yn = ((Y.float() - self.y_mean) / self.y_std).contiguous()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        losses = self.net.fit(Xn, Yn, steps=steps, batch=batch, lr=lr, seed=seed)
        torch.cuda.synchronize()
        return losses, time.perf_counter() - t0

    def predict(self, X: torch.Tensor) -> torch.Tensor:
        Xn = (X.float().reshape(-1, self.widths[0]) * self.x_scale).contiguous()
        return self.net.forward(Xn) * self.y_std + self.y_mean

    def cost_and_grad(self, c: torch.Tensor, w: torch.Tensor):
        """J_sur = sum_n w_n exp(y_n) and its gradient with respect to c (one coefficient vector)."""
        Xn = (c.float().reshape(1, -1) * self.x_scale).contiguous()
        z = self.net.forward(Xn)
        e = torch.exp(z * self.y_std + self.y_mean) * w
        g_x = self.net.backward((e * self.y_std).contiguous(), param_grads=False, input_grad=True)
        return e.sum(), (g_x * self.x_scale).reshape(-1)


class ControlProblem:
    """True J(c) = trapezoid(ee, dt) and dJ/dc through the fused forward and adjoint kernels."""

    def __init__(self, setup: ControlSetup, dtype=torch.float32):
        self.setup = setup
        self.plan = Plan(setup.mesh, setup.dt, setup.f_eq, dtype=dtype)
        dev = self.plan.device
        self.B = torch.tensor(fourier_basis(setup.mesh.xs, setup.k0, setup.n_modes), dtype=dtype,
                              device=dev)
        self.f_iv = torch.tensor(np.asarray(setup.f_iv), dtype=torch.float64, device=dev)
        self.w = torch.tensor(trapezoid_weights(setup.n_steps, setup.dt), dtype=dtype, device=dev)
        self.evals = 0

    def value_and_grad(self, c: torch.Tensor):
        T = self.setup.n_steps
        H = (self.B @ c.to(self.B.dtype)).contiguous()
        out = self.plan.forward(self.f_iv, H, T, record_history=False, want_tape=True,
                                want_f_final=False)
        J = (out["ee_hist"] * self.w).sum()
        _, g_H = self.plan.backward(H, T, out["tape"], out["every"], g_ee_hist=self.w)
        self.evals += 1
        return J, (self.B.T @ g_H)


def adam_loop(fun, c0: torch.Tensor, lr: float, max_iters: int, stop,
              b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8):
    """Adam (Kingma & Ba) on ``fun(c) -> (J, dJ/dc)``; ``stop(history)`` is checked after each
    evaluation. Returns (best c, best J, history of J)."""
    c = c0.clone().float()
    m = torch.zeros_like(c)
    v = torch.zeros_like(c)
    hist = []
    best = (float("inf"), c.clone())
    for t in range(1, max_iters + 1):
        J, g = fun(c)
        Jf = float(J)
        hist.append(Jf)
        if Jf < best[0]:
            best = (Jf, c.clone())
        if stop(hist):
            break
        g = g.float()
        m = b1 * m + (1 - b1) * g
        v = b2 * v + (1 - b2) * g * g
        c = c - lr * (m / (1 - b1 ** t)) / ((v / (1 - b2 ** t)).sqrt() + eps)
    return best[1], best[0], hist


def optimize_plain(problem: ControlProblem, c0, lr: float = 1e-3, max_iters: int = 4000,
                   window: int = 20, rtol: float = 1e-4):
    """Adam with the true gradient until J stops improving: the best J of the last ``window``
    evaluations is not below (1 - rtol) times the best before them."""
    def stop(h):
        if len(h) <= 2 * window:
            return False
        return min(h[-window:]) > min(h[:-window]) * (1 - rtol)
    problem.evals = 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    c, J, hist = adam_loop(problem.value_and_grad, c0, lr, max_iters, stop)
    torch.cuda.synchronize()
    return {"c": c, "J": J, "seconds": time.perf_counter() - t0, "evals": problem.evals,
            "history": hist}


def evals_to_reach(history, target: float) -> int | None:
    h = np.asarray(history)
    hit = np.nonzero(h <= target)[0]
    return int(hit[0]) + 1 if hit.size else None


class SurrogateSearch:
    """Adam on the surrogate's J = sum_n w_n exp(y_n(c)) for one coefficient vector, run as one
    single-CTA launch per search (``vp_mlp_search``: warp GEMVs on the network's BF16 weights,
    best-iterate tracking on the device, no host synchronisation)."""

    def __init__(self, sur: Surrogate, w: torch.Tensor, lr: float, b1: float = 0.9,
                 b2: float = 0.999, eps: float = 1e-8):
        from . import _capi
        self.sur = sur
        self.lib = _capi.load()
        dev = sur.net.device
        self.w = w.float().to(dev).reshape(-1).contiguous()
        self.y_mean = sur.y_mean.float().to(dev).contiguous()
        self.y_std = sur.y_std.float().to(dev).contiguous()
        self.lr, self.b1, self.b2, self.eps = lr, b1, b2, eps
        self.best_c = torch.zeros(sur.widths[0], device=dev)
        self.best_J = torch.zeros(1, device=dev)

    def run(self, c0: torch.Tensor, iters: int) -> torch.Tensor:
        from . import _capi
        from .plan import _stream_handle
        c0 = c0.float().reshape(-1).contiguous().to(self.best_c.device)
        _capi.check(self.lib.vp_mlp_search(
            self.sur.net._h, _capi.ptr(c0), int(iters), float(self.lr), float(self.b1), float(self.b2),
            float(self.eps), float(self.sur.x_scale), _capi.ptr(self.y_mean), _capi.ptr(self.y_std),
            _capi.ptr(self.w), _capi.ptr(self.best_c), _capi.ptr(self.best_J),
            _stream_handle(self.best_c.device)))
        return self.best_c.clone()


def optimize_warm(problem: ControlProblem, sur: Surrogate, c0, J_target: float,
                  lr_sur: float = 3e-3, lr: float = 1e-3, sur_iters: int = 150,
                  max_iters: int = 4000, search: SurrogateSearch | None = None):
    """Minimise the surrogate's J from c0, then refine with the true gradient (Adam, step size
    ``lr``) until J <= J_target. ``seconds`` covers both phases (the surrogate's training is
    separate)."""
    if search is None:
        search = SurrogateSearch(sur, problem.w, lr_sur)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    c_sur = search.run(c0, sur_iters)
    torch.cuda.synchronize()
    t_sur = time.perf_counter() - t0
    problem.evals = 0
    c, J, hist = adam_loop(problem.value_and_grad, c_sur, lr, max_iters,
                           lambda h: h[-1] <= J_target)
    torch.cuda.synchronize()
    return {"c": c, "J": J, "seconds": time.perf_counter() - t0, "surrogate_seconds": t_sur,
            "evals": problem.evals, "history": hist, "reached": J <= J_target}


def c5_setup(nx: int = 256, nv: int = 256, n_steps: int = 100, n_modes: int = 16, eps: float = 1e-3):
    """Two-stream set-up of the surrogate benchmark: L_x = 10 pi, v in [-6, 6), mu = 2.4,
    perturbation eps cos(0.2 x), dt 0.05."""
    from .mesh import make_mesh
    from .workloads import two_stream
    m = make_mesh(10.0 * np.pi, 6.0, nx, nv)
    f_eq, f_iv = two_stream(m, eps=eps)
    return ControlSetup(m, 0.05, n_steps, f_eq, f_iv, n_modes)


def run_comparison(setup: ControlSetup, n_samples: int, coeff_std: float, train_steps: int,
                   seeds, batch: int = 1024, sur_iters: int = 150, lr_sur: float = 3e-3,
                   lr: float = 1e-3, lr_refine: float | None = None, data_seed: int = 0, net_seed: int = 1,
                   tol: float = 0.01):
    """Data generation, training, then plain vs warm-started control from random initial
    coefficients (standard deviation ``coeff_std``, one per seed). The plain loop uses Adam with
    step size ``lr``; the warm start's true-gradient refinement uses ``lr_refine`` (default
    ``lr``). Returns a summary dict."""
    X, Y, data = generate_dataset(setup, n_samples, coeff_std, seed=data_seed)
    n_hold = max(1, n_samples // 10)
    sur = Surrogate(setup.n_inputs, setup.n_steps, max_batch=max(256, n_samples), seed=net_seed)
    losses, t_train = sur.fit(X[:-n_hold], Y[:-n_hold], steps=train_steps, batch=batch)
    hold = float((sur.predict(X[-n_hold:]) - Y[-n_hold:]).abs().mean())
    hold_base = float((Y[:-n_hold].mean(0) - Y[-n_hold:]).abs().mean())
    prob = ControlProblem(setup)
    search = SurrogateSearch(sur, prob.w, lr_sur)
    runs = []
    for seed in seeds:
        c0 = torch.tensor(coeff_std * np.random.default_rng(seed).standard_normal(setup.n_inputs),
                          dtype=torch.float32, device=prob.plan.device)
        plain = optimize_plain(prob, c0, lr=lr)
        target = (1 + tol) * plain["J"]
        warm = optimize_warm(prob, sur, c0, target, lr_sur=lr_sur, lr=lr if lr_refine is None else lr_refine,
                             sur_iters=sur_iters, search=search)
        runs.append({"seed": int(seed), "J0": plain["history"][0], "J_star": plain["J"],
                     "plain_evals": plain["evals"], "plain_seconds": plain["seconds"],
                     "plain_evals_to_target": evals_to_reach(plain["history"], target),
                     "warm_J": warm["J"], "warm_reached": bool(warm["reached"]),
                     "warm_evals": warm["evals"], "warm_seconds": warm["seconds"],
                     "warm_surrogate_seconds": warm["surrogate_seconds"],
                     "time_ratio": warm["seconds"] / plain["seconds"]})
    return {"data": data, "train_seconds": t_train, "train_steps": train_steps,
            "final_loss": float(np.mean(losses[-20:])), "holdout_mae_log_ee": hold,
            "holdout_mae_mean_predictor": hold_base, "runs": runs,
            "mlp_status": sur.net.status()}
