"""The warm-start network's device kernels against the CPU restatement
(oracle/mlp_ref.py): forward, loss and gradient (FP32 device vs FP64 oracle,
relative tolerance 1e-4 on the gradient norm and 2e-4 per output), and one
short training run that must lower the loss."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SMALL = (4, 32, 48, 24)


def _data(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, (n, 4)).astype(np.float32)
    t = np.stack([np.sin(1.3 * x[:, 0] + k * 0.2) * np.cos(x[:, 1] - 0.1 * k) + 0.3 * x[:, 2] * x[:, 3]
                  for k in range(SMALL[3])], axis=1).astype(np.float32)
    return x, t


def test_forward_and_gradient_match_oracle(gpu_ctx):
    from atlas12_b200.warmstart import MLP
    import mlp_ref
    m = MLP(gpu_ctx, shape=SMALL, seed=3)
    p32 = m.params()
    assert p32.size == m.nparam and np.all(np.isfinite(p32)), (p32.size, m.nparam)
    p = p32.astype(np.float64)
    x, t = _data(77, 1)
    y = m.forward(x)
    _, _, yr = mlp_ref.forward(p, x, SMALL)
    assert np.all(np.isfinite(yr)), (np.isfinite(p).all(), np.isfinite(x).all(), mlp_ref.__file__)
    np.testing.assert_allclose(y, yr, rtol=2e-4, atol=2e-5)
    loss, g = m.loss_grad(x, t)
    lr, gr = mlp_ref.loss_grad(p, x, t, SMALL)
    assert abs(loss - lr) <= 1e-4 * lr
    assert np.linalg.norm(g - gr) <= 1e-4 * np.linalg.norm(gr)
    m.close()


def test_training_lowers_loss(gpu_ctx):
    from atlas12_b200.warmstart import MLP
    m = MLP(gpu_ctx, shape=SMALL, seed=5)
    x, t = _data(512, 2)
    l0, _ = m.loss_grad(x, t)
    hist = m.train(x, t, epochs=200, batch=64, lr=3e-3, seed=9)
    l1, _ = m.loss_grad(x, t)
    assert np.all(np.isfinite(hist))
    assert l1 < 0.1 * l0, (l0, l1)
    m.close()
