"""CPU restatement of the surrogate MLP's arithmetic (TEST INFRASTRUCTURE ONLY).

Checks the tensor-core kernels of ``warp_vp_solver_b200/csrc/vp_mlp.cu``: the same network
(widths[0] -> ... -> widths[-1], GELU in erf form between layers, none on the output), the same
packing of parameters (per layer W_l [out, in] row-major, then b_l), and, with
``emulate_bf16=True``, the same rounding points: every GEMM operand is rounded to bfloat16
(round to nearest even) and products are accumulated exactly (float64 here, float32 on the GPU);
bias, GELU, GELU' and the loss stay in full precision. With ``emulate_bf16=False`` it is the plain
float64 network, used to check the backward formulas against finite differences.

Adam follows Kingma & Ba (2015), Algorithm 1, with bias corrections 1 - beta^t.
"""

from __future__ import annotations

import numpy as np
from scipy.special import erf


def bf16(x) -> np.ndarray:
    """Round to bfloat16 (nearest even), returned as float64."""
    u = np.ascontiguousarray(np.asarray(x, dtype=np.float32)).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def param_count(widths) -> int:
    return int(sum(widths[i] * widths[i + 1] + widths[i + 1] for i in range(len(widths) - 1)))


def unpack(params, widths):
    p = np.asarray(params, dtype=np.float64)
    out, off = [], 0
    for i in range(len(widths) - 1):
        k, n = widths[i], widths[i + 1]
        W = p[off:off + n * k].reshape(n, k)
        off += n * k
        b = p[off:off + n]
        off += n
        out.append((W, b))
    return out


def init_params(widths, seed: int) -> np.ndarray:
    """U(-1/sqrt(fan_in), 1/sqrt(fan_in)) for weights and biases (the torch.nn.Linear default)."""
    rng = np.random.default_rng(seed)
    chunks = []
    for i in range(len(widths) - 1):
        k, n = widths[i], widths[i + 1]
        a = 1.0 / np.sqrt(k)
        chunks += [rng.uniform(-a, a, n * k), rng.uniform(-a, a, n)]
    return np.concatenate(chunks).astype(np.float32)


def forward(params, widths, X, emulate_bf16=True):
    r = bf16 if emulate_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    layers = unpack(params, widths)
    a = r(X)
    cache = {"A": [a], "Z": []}
    for i, (W, b) in enumerate(layers):
        z = a @ r(W).T + b
        if i == len(layers) - 1:
            cache["Y"] = z
            return z, cache
        cache["Z"].append(z)
        a = r(gelu(z))
        cache["A"].append(a)
    raise AssertionError("unreachable")


def backward(params, widths, cache, g_Y, emulate_bf16=True, input_grad=False):
    """Parameter gradients (packed like the parameters) and optionally the input cotangent."""
    r = bf16 if emulate_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    layers = unpack(params, widths)
    d = np.asarray(g_Y, dtype=np.float64)
    grads = [None] * len(layers)
    g_X = None
    for i in range(len(layers) - 1, -1, -1):
        W, _ = layers[i]
        db = d.sum(axis=0)
        dW = r(d).T @ cache["A"][i]
        grads[i] = (dW, db)
        if i > 0 or input_grad:
            da = r(d) @ r(W)
            if i > 0:
                d = da * gelu_grad(cache["Z"][i - 1])
            else:
                g_X = da
    flat = np.concatenate([np.concatenate([dW.ravel(), db]) for dW, db in grads])
    return flat, g_X


def mse_backward(params, widths, cache, target, emulate_bf16=True):
    Y = cache["Y"]
    e = Y - np.asarray(target, dtype=np.float64)
    loss = float((e * e).mean())
    g, _ = backward(params, widths, cache, 2.0 * e / e.size, emulate_bf16)
    return loss, g


def adam(p, g, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step at step number t (1-based); returns (p, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    p = p - lr * (m / (1 - b1 ** t)) / (np.sqrt(v / (1 - b2 ** t)) + eps)
    return p, m, v
