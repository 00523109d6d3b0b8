"""The GPU MLP (tensor-core BF16 forward, backward, Adam) against its CPU
checker tests/mlp_ref.py: same bf16 roundings, FP64 accumulation there.

Bars: forward outputs within 1e-2 relative (max over the batch, scaled by
the largest output); the gradient within 2e-2 relative L2 overall and per
layer -- FP32 accumulation order and an occasional different bf16 rounding
of an activation are the only differences."""
import numpy as np
import pytest

import lbib
import mlp_ref

pytestmark = pytest.mark.gpu


def _data(rng, batch, widths):
    import torch
    X = rng.normal(0, 1, (batch, widths[0])).astype(np.float32)
    T = rng.normal(0, 0.5, (batch, widths[-1])).astype(np.float32)
    return X, T, torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()


@pytest.mark.parametrize("widths,batch", [([5, 32, 32, 24], 64), ([5, 256, 256, 256, 256, 192], 1024),
                                          ([3, 40, 17], 50)])
def test_forward_and_gradient_match_cpu(gpu, widths, batch):
    rng = np.random.default_rng(1)
    with lbib.MLP(widths, max_batch=batch, seed=3) as net:
        p = net.params()
        p += rng.normal(0, 0.02, p.size).astype(np.float32)   # non-zero biases too
        net.set_params(p)
        np.testing.assert_array_equal(net.params(), p)
        X, T, Xd, Td = _data(rng, batch, widths)
        Y = net.forward(Xd).cpu().numpy()
        g, loss = net.gradient(Xd, Td)
    Yr, _, _ = mlp_ref.forward(p, widths, X)
    assert np.max(np.abs(Y - Yr)) <= 1e-2 * np.max(np.abs(Yr))
    lr, gr = mlp_ref.loss_and_grad(p, widths, X, T)
    assert abs(loss - lr) <= 1e-2 * lr
    assert np.linalg.norm(g - gr) <= 2e-2 * np.linalg.norm(gr)
    i = 0
    for l in range(len(widths) - 1):
        n = widths[l] * widths[l + 1] + widths[l + 1]
        a, b = g[i:i + n], gr[i:i + n]
        assert np.linalg.norm(a - b) <= 2e-2 * np.linalg.norm(b), l
        i += n


def test_adam_training_fits_a_smooth_map(gpu):
    import torch
    rng = np.random.default_rng(4)
    widths = [5, 64, 64, 12]
    X = rng.uniform(-1, 1, (4096, 5)).astype(np.float32)
    M = rng.normal(0, 1, (5, 12))
    T = np.tanh(X @ M).astype(np.float32)
    Xd, Td = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    with lbib.MLP(widths, max_batch=512, seed=7) as net:
        first = net.train_step(Xd[:512], Td[:512], 3e-3, want_loss=True)
        for it in range(600):
            k = (it % 8) * 512
            net.train_step(Xd[k:k + 512], Td[k:k + 512], 3e-3)
        last = net.train_step(Xd[:512], Td[:512], 3e-3, want_loss=True)
    assert last < 0.05 * first, (first, last)


def test_training_on_fresh_gathered_batches(gpu):
    """Batches gathered by torch just before each step (temporaries on
    torch's stream) must be what the MLP trains on."""
    import torch
    rng = np.random.default_rng(5)
    X = rng.uniform(-1, 1, (8192, 5)).astype(np.float32)
    T = np.tanh(X @ rng.normal(0, 1, (5, 24))).astype(np.float32)
    Xd, Td = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    with lbib.MLP([5, 64, 64, 24], max_batch=1024, seed=7) as net:
        first = None
        for it in range(800):
            idx = torch.randint(0, 8192, (1024,), device="cuda", generator=g)
            loss = net.train_step(Xd[idx].contiguous(), Td[idx].contiguous(), 3e-3, want_loss=it in (0, 799))
            if it == 0:
                first = loss
        assert loss < 0.02 * first, (first, loss)
