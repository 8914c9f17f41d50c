"""Tensor-core MLP kernels (tcgen05, BF16 in / FP32 accumulate) against a torch FP32 reference of
the same GEMMs and against the CPU oracle of the network (oracle/mlp_oracle.py).

Bars (max-norm relative error): a single GEMM vs torch FP32 on the same BF16 operands 1e-5 (only
the summation order differs); the network vs the oracle 1e-2 on outputs and gradients (operands
are rounded to BF16 at the same points, but an FP32-vs-FP64 difference can flip one rounding,
about 2^-8 relative on that element).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import mlp_oracle as MO
from warp_vp_solver_b200 import _capi
from warp_vp_solver_b200.mlp import MLP

pytestmark = pytest.mark.gpu

WIDTHS = [32, 256, 256, 100]


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _gemm(A, B, bias=None, act=0, aux=None, want16=True):
    lib = _capi.load()
    M, K = A.shape
    N = B.shape[0]
    np8 = (N + 7) // 8 * 8
    mp8 = (M + 7) // 8 * 8
    C32 = torch.full((M, N), float("nan"), device="cuda")
    C16 = torch.full((M, np8), 7.0, dtype=torch.bfloat16, device="cuda") if want16 else None
    C16T = torch.full((N, mp8), 7.0, dtype=torch.bfloat16, device="cuda") if want16 else None
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    _capi.check(lib.vp_gemm_bf16(
        A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0), M, N, K,
        _capi.ptr(bias), act, _capi.ptr(aux), aux.stride(0) if aux is not None else 0,
        C32.data_ptr(), N, _capi.ptr(C16), np8, _capi.ptr(C16T), mp8, err.data_ptr(),
        torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return C32, C16, C16T


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (200, 100, 96), (1, 32, 256), (333, 72, 136),
                                   (4096, 256, 256), (64, 256, 4096)])
def test_gemm_matches_torch_fp32(M, N, K):
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    C32, C16, C16T = _gemm(A, B)
    ref = A.float() @ B.float().T
    assert rel(C32.cpu(), ref.cpu()) < 1e-5
    assert torch.equal(C16[:, :N], C32.to(torch.bfloat16))
    assert torch.equal(C16T[:, :M], C16[:, :N].T)
    # padding columns are written as zero
    assert (C16[:, N:] == 0).all() and (C16T[:, M:] == 0).all()


def test_gemm_epilogues_match_torch():
    M, N, K = 260, 192, 128
    g = torch.Generator(device="cuda").manual_seed(1)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = (0.1 * torch.randn(N, K, device="cuda", generator=g)).to(torch.bfloat16)
    bias = torch.randn(N, device="cuda", generator=g)
    z = A.float() @ B.float().T + bias
    C32, C16, _ = _gemm(A, B, bias=bias, act=1)
    assert rel(C32.cpu(), torch.nn.functional.gelu(z).cpu()) < 1e-5
    aux = torch.randn(M, N, device="cuda", generator=g)
    C32, _, _ = _gemm(A, B, bias=bias, act=2, aux=aux)
    x = aux.double()
    dg = 0.5 * (1 + torch.erf(x / np.sqrt(2))) + x * torch.exp(-0.5 * x * x) / np.sqrt(2 * np.pi)
    assert rel(C32.cpu(), (z.double() * dg).cpu()) < 1e-5


@pytest.mark.parametrize("M", [203, 512])
def test_mlp_forward_and_gradients_match_oracle(M):
    net = MLP(WIDTHS, max_batch=1024, seed=3)
    rng = np.random.default_rng(M)
    X = rng.standard_normal((M + 17, 32)).astype(np.float32)
    T = rng.standard_normal((M + 17, 100)).astype(np.float32)
    rows = rng.permutation(M + 17)[:M].astype(np.int32)
    p = net.get_params().cpu().numpy()
    Xt, Tt = torch.tensor(X, device="cuda"), torch.tensor(T, device="cuda")
    rt = torch.tensor(rows, device="cuda")
    Y = net.forward(Xt, rt).cpu().numpy()
    Yo, cache = MO.forward(p, WIDTHS, X[rows])
    assert rel(Y, Yo) < 1e-2
    loss = net.train_step(Xt, Tt, rt).item()
    g = net.get_grads().cpu().numpy()
    lo, go = MO.mse_backward(p, WIDTHS, cache, T[rows])
    assert abs(loss - lo) / lo < 1e-3
    assert rel(g, go) < 1e-2
    # per layer as well, so that a small layer's gradient is not hidden by a large one
    off = 0
    for i in range(len(WIDTHS) - 1):
        n = WIDTHS[i] * WIDTHS[i + 1] + WIDTHS[i + 1]
        assert rel(g[off:off + n], go[off:off + n]) < 1e-2, f"layer {i}"
        off += n
    # input cotangent through vp_mlp_backward
    gY = rng.standard_normal((M, 100)).astype(np.float32)
    net.forward(Xt, rt)
    gX = net.backward(torch.tensor(gY, device="cuda"), param_grads=True, input_grad=True).cpu().numpy()
    gp, gXo = MO.backward(p, WIDTHS, cache, gY, input_grad=True)
    assert rel(gX, gXo) < 1e-2
    assert rel(net.get_grads().cpu().numpy(), gp) < 1e-2
    assert net.status() == 0


def test_adam_step_matches_oracle():
    net = MLP(WIDTHS, max_batch=256, seed=5)
    rng = np.random.default_rng(0)
    X = torch.tensor(rng.standard_normal((256, 32)), dtype=torch.float32, device="cuda")
    T = torch.tensor(rng.standard_normal((256, 100)), dtype=torch.float32, device="cuda")
    p = net.get_params().cpu().numpy().astype(np.float64)
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    for t in range(1, 4):
        net.train_step(X, T)
        g = net.get_grads().cpu().numpy().astype(np.float64)
        net.adam(lr=1e-3)
        p, m, v = MO.adam(p, g, m, v, t, 1e-3)
        got = net.get_params().cpu().numpy()
        assert rel(got, p) < 1e-6
        p = got.astype(np.float64)   # continue from the device's float32 parameters


def test_fit_graph_replay_is_deterministic_and_learns():
    rng = np.random.default_rng(1)
    X = rng.standard_normal((2048, 32)).astype(np.float32)
    Wt = rng.standard_normal((32, 100)) / np.sqrt(32)
    T = np.sin(X @ Wt).astype(np.float32)
    a = MLP(WIDTHS, max_batch=256, seed=7)
    la = a.fit(X, T, steps=300, batch=256, lr=1e-3, seed=0, use_graph=True)
    b = MLP(WIDTHS, max_batch=256, seed=7)
    lb = b.fit(X, T, steps=300, batch=256, lr=1e-3, seed=0, use_graph=False)
    np.testing.assert_array_equal(la, lb)
    assert torch.equal(a.get_params(), b.get_params())
    assert la[-20:].mean() < 0.5 * la[:5].mean()
    assert a.status() == 0 and b.status() == 0
