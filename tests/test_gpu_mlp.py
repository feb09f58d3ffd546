"""Warm-start network kernels on the GPU: the tcgen05 GEMM against torch's
FP32 matmul of the same BF16 operands, and the network's forward pass,
gradients and first Adam step against the CPU oracle (FP64 with the GPU's
BF16 roundings emulated)."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))


@pytest.mark.parametrize("m,n,k", [(128, 16, 16), (128, 128, 64), (256, 256, 256), (128, 512, 256),
                                   (512, 256, 256), (256, 16, 256), (384, 128, 80), (128, 32, 512)])
def test_gemm_matches_torch(m, n, k):
    import torch
    from ekpnp.mlp import gemm_bf16
    g = torch.Generator(device="cuda").manual_seed(m * 7 + n * 3 + k)
    a = torch.randn(m, k, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(n, k, device="cuda", generator=g).to(torch.bfloat16)
    c = torch.full((m, n), float("nan"), device="cuda")
    gemm_bf16(a, b, c)
    ref = a.double() @ b.double().T
    err = (c.double() - ref).abs().max().item()
    # FP32 accumulation of k products of magnitude ~1
    assert err <= 2e-6 * k, err


def test_gemm_strided_operands():
    import torch
    from ekpnp.mlp import gemm_bf16
    g = torch.Generator(device="cuda").manual_seed(5)
    big_a = torch.randn(256, 96, device="cuda", generator=g).to(torch.bfloat16)
    big_b = torch.randn(64, 96, device="cuda", generator=g).to(torch.bfloat16)
    a, b = big_a[:, 16:80], big_b[:, 16:80]   # lda = ldb = 96, k = 64
    c = torch.zeros(256, 64, device="cuda")
    gemm_bf16(a, b, c)
    ref = a.double() @ b.double().T
    assert (c.double() - ref).abs().max().item() <= 2e-6 * 64


def batch(seed, B=256):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, (B, 4)).astype(np.float32)
    s = np.linspace(0, 1, 128)
    t = np.concatenate([np.sin(np.pi * s[None, :] * (1 + 0.5 * x[:, :1])) * (1 + 0.3 * x[:, 1:2]),
                        np.tanh(4 * x[:, 2:3] * s[None, :]), np.cos(3 * s[None, :] + x[:, 3:4]),
                        x[:, :1] * s[None, :] ** 2], axis=1).astype(np.float32)
    return x, t


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_forward_and_gradients_match_oracle():
    import ekpnp.mlp as em
    import mlp_oracle as mo
    x, t = batch(1)
    with em.Mlp(batch=256, seed=3) as net:
        p = net.params
        y = net.forward(x)
        g, loss = net.gradients(x, t)
    y_ref, _ = mo.forward(p.astype(np.float64), x.astype(np.float64))
    assert rel(y, y_ref) < 5e-3
    loss_ref, g_ref = mo.loss_and_gradients(p.astype(np.float64), x.astype(np.float64), t.astype(np.float64))
    assert abs(loss - loss_ref) <= 1e-3 * loss_ref
    for l, ((ws, _, bs), (wr, br)) in enumerate(zip(em.layer_slices(), zip(*[iter(range(8))] * 2))):
        assert rel(g[ws], g_ref[ws]) < 2e-2, ("W", l, rel(g[ws], g_ref[ws]))
        assert rel(g[bs], g_ref[bs]) < 2e-2, ("b", l, rel(g[bs], g_ref[bs]))


def test_first_adam_step_matches_oracle():
    import ekpnp.mlp as em
    import mlp_oracle as mo
    x, t = batch(2)
    lr = 1e-3
    with em.Mlp(batch=256, seed=4) as net:
        p0 = net.params
        net.set_data(x, t)       # one batch: the epoch permutation only reorders rows
        loss = net.train(1, lr)
        p1 = net.params
    _, g_ref = mo.loss_and_gradients(p0.astype(np.float64), x.astype(np.float64), t.astype(np.float64))
    # first Adam step: m_hat = g, v_hat = g^2, so p1 = p0 - lr g / (|g| + 1e-8)
    want = p0 - lr * g_ref / (np.abs(g_ref) + 1e-8)
    big = np.abs(g_ref) > 1e-3 * np.abs(g_ref).max()
    assert np.abs(p1 - want)[big].max() < 1e-6 + 1e-3 * lr
    assert loss[0] > 0


def test_training_reduces_loss_and_counts_launches():
    import ekpnp.mlp as em
    xs, ts = zip(*[batch(10 + i) for i in range(8)])
    x, t = np.concatenate(xs), np.concatenate(ts)
    with em.Mlp(batch=256, seed=5) as net:
        net.set_data(x, t)
        l0 = net.launches
        loss = net.train(600, 2e-3)
        assert net.launches - l0 == 600 * 16
        y = net.forward(x[:300])
    assert np.all(np.isfinite(loss))
    assert loss[-20:].mean() < 0.05 * loss[:5].mean()
    assert float(np.mean((y - t[:300]) ** 2)) < 0.1 * loss[:5].mean()
