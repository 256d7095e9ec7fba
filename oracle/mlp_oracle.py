"""TEST INFRASTRUCTURE ONLY — float64 numpy restatement of the firing predictor's
MLP (9 -> 64 -> 64 -> 1, ReLU) and of its mean-squared-error gradient, the CPU
check for the engine's forward and backward kernels. Parameter layout:
W1[64][9], b1[64], W2[64][64], b2[64], W3[64], b3."""
import numpy as np

IN, H = 9, 64


def unpack(p):
    p = np.asarray(p, np.float64)
    o = 0
    W1 = p[o:o + H * IN].reshape(H, IN); o += H * IN
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + H]; o += H
    b3 = p[o]
    return W1, b1, W2, b2, W3, b3


def forward(p, x):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    x = np.asarray(x, np.float64)
    h1 = np.maximum(x @ W1.T + b1, 0.0)
    h2 = np.maximum(h1 @ W2.T + b2, 0.0)
    return h2 @ W3 + b3


def loss_and_grad(p, x, y):
    """Mean squared error over the samples and its gradient (manual backprop)."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    n = x.shape[0]
    z1 = x @ W1.T + b1
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0.0)
    out = h2 @ W3 + b3
    e = out - y
    loss = float(np.mean(e * e))
    dy = 2.0 * e / n
    gW3 = h2.T @ dy
    gb3 = dy.sum()
    dz2 = np.outer(dy, W3) * (z2 > 0)
    gW2 = dz2.T @ h1
    gb2 = dz2.sum(0)
    dz1 = (dz2 @ W2) * (z1 > 0)
    gW1 = dz1.T @ x
    gb1 = dz1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])
    return loss, g
