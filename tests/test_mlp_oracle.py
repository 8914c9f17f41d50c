"""The MLP oracle (CPU restatement of the surrogate network's arithmetic) against finite
differences and torch's Adam; bfloat16 rounding against torch's conversion."""

from __future__ import annotations

import numpy as np
import torch

import mlp_oracle as MO


def test_bf16_rounding_matches_torch():
    x = np.random.default_rng(0).standard_normal(4096).astype(np.float32) * 10
    ref = torch.tensor(x).to(torch.bfloat16).to(torch.float64).numpy()
    np.testing.assert_array_equal(MO.bf16(x), ref)


def test_backward_matches_central_differences():
    widths = [5, 7, 6, 3]
    p = MO.init_params(widths, 1).astype(np.float64)
    rng = np.random.default_rng(2)
    X = rng.standard_normal((4, 5))
    T = rng.standard_normal((4, 3))
    _, cache = MO.forward(p, widths, X, emulate_bf16=False)
    _, g = MO.mse_backward(p, widths, cache, T, emulate_bf16=False)

    def loss(q):
        Y, _ = MO.forward(q, widths, X, emulate_bf16=False)
        return ((Y - T) ** 2).mean()

    h = 1e-6
    fd = np.array([(loss(p + h * e) - loss(p - h * e)) / (2 * h) for e in np.eye(p.size)])
    np.testing.assert_allclose(g, fd, rtol=1e-6, atol=1e-9)


def test_input_gradient_matches_central_differences():
    widths = [4, 8, 2]
    p = MO.init_params(widths, 3).astype(np.float64)
    X = np.random.default_rng(4).standard_normal((3, 4))
    gY = np.random.default_rng(5).standard_normal((3, 2))
    _, cache = MO.forward(p, widths, X, emulate_bf16=False)
    _, gX = MO.backward(p, widths, cache, gY, emulate_bf16=False, input_grad=True)
    h = 1e-6
    fd = np.zeros_like(X)
    for i in range(X.shape[0]):
        for j in range(X.shape[1]):
            e = np.zeros_like(X)
            e[i, j] = h
            fd[i, j] = ((MO.forward(p, widths, X + e, False)[0] - MO.forward(p, widths, X - e, False)[0])
                        * gY).sum() / (2 * h)
    np.testing.assert_allclose(gX, fd, rtol=1e-6, atol=1e-9)


def test_adam_matches_torch():
    rng = np.random.default_rng(6)
    p0 = rng.standard_normal(10)
    grads = rng.standard_normal((5, 10))
    t = torch.tensor(p0, requires_grad=True)
    opt = torch.optim.Adam([t], lr=1e-2, betas=(0.9, 0.999), eps=1e-8)
    p, m, v = p0.copy(), np.zeros(10), np.zeros(10)
    for k in range(5):
        opt.zero_grad()
        t.grad = torch.tensor(grads[k])
        opt.step()
        p, m, v = MO.adam(p, grads[k], m, v, k + 1, 1e-2)
    np.testing.assert_allclose(p, t.detach().numpy(), rtol=1e-12, atol=1e-12)
