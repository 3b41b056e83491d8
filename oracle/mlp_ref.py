"""numpy restatement of the cost-model MLP (test infrastructure only).

Same parameter layout as the engine's kernels: W1[H][in] b1[H] W2[H][H] b2[H]
W3[H] b3, ReLU hidden layers, loss = mean((y - t)^2).  Used to check the
GPU forward pass and the GPU gradient of every parameter.
"""
import numpy as np

H = 64


def unpack(p, nin):
    o = 0
    W1 = p[o:o + H * nin].reshape(H, nin); o += H * nin
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + H]; o += H
    b3 = p[o]; o += 1
    assert o == p.size
    return W1, b1, W2, b2, W3, b3


def forward(p, X):
    p = p.astype(np.float64)
    X = X.astype(np.float64)
    W1, b1, W2, b2, W3, b3 = unpack(p, X.shape[1])
    a1 = X @ W1.T + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0)
    y = h2 @ W3 + b3
    return y, (a1, h1, a2, h2)


def loss_grad(p, X, t):
    n, nin = X.shape
    W1, b1, W2, b2, W3, b3 = unpack(p.astype(np.float64), nin)
    y, (a1, h1, a2, h2) = forward(p, X)
    e = y - t.astype(np.float64)
    loss = np.mean(e * e)
    dy = 2 * e / n
    gW3 = h2.T @ dy
    gb3 = dy.sum()
    dh2 = np.outer(dy, W3) * (a2 > 0)
    gW2 = dh2.T @ h1
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ W2) * (a1 > 0)
    gW1 = dh1.T @ X.astype(np.float64)
    gb1 = dh1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])
    return loss, g
