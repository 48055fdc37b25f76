"""CPU restatement of the warm-start network (test infrastructure only).

The checker for atlas12_b200/csrc/mlp.cu: the same dense tanh MLP
(nin -> nh1 -> nh2 -> nout, W stored [out][in] row-major, one flat parameter
vector [W1, b1, W2, b2, W3, b3]) with its mean-squared-error loss, forward
and backward in float64 numpy.  Only tests import it.
"""
import numpy as np


def split(params, nin, nh1, nh2, nout):
    p = np.asarray(params, dtype=np.float64)
    shapes = [(nh1, nin), (nh1,), (nh2, nh1), (nh2,), (nout, nh2), (nout,)]
    out, o = [], 0
    for s in shapes:
        n = int(np.prod(s))
        out.append(p[o:o + n].reshape(s))
        o += n
    assert o == p.size
    return out


def forward(params, x, shape):
    W1, b1, W2, b2, W3, b3 = split(params, *shape)
    x = np.asarray(x, dtype=np.float64)
    h1 = np.tanh(x @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    return h1, h2, h2 @ W3.T + b3


def loss_grad(params, x, t, shape):
    """Mean squared error over samples and outputs, and its gradient."""
    W1, b1, W2, b2, W3, b3 = split(params, *shape)
    x = np.asarray(x, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    h1, h2, y = forward(params, x, shape)
    n = y.size
    loss = np.sum((y - t) ** 2) / n
    dy = 2.0 * (y - t) / n
    gW3, gb3 = dy.T @ h2, dy.sum(0)
    d2 = (dy @ W3) * (1.0 - h2 ** 2)
    gW2, gb2 = d2.T @ h1, d2.sum(0)
    d1 = (d2 @ W2) * (1.0 - h1 ** 2)
    gW1, gb1 = d1.T @ x, d1.sum(0)
    g = np.concatenate([a.ravel() for a in (gW1, gb1, gW2, gb2, gW3, gb3)])
    return loss, g
