"""FP64 numpy restatement of the learned indicator's network, loss and gradient.

TEST INFRASTRUCTURE ONLY (the checker of the CUDA training kernels): same architecture and packing
as include/nemo_gpu.h -- x = feat/10 + 1, h1 = SiLU(W1 x + b1), h2 = SiLU(W2 h1 + b2),
alpha = amax * sigmoid(W3 . h2 + b3), loss = mean (alpha - target)^2.
"""
import numpy as np

NW = 32 * 12 + 32 + 32 * 32 + 32 + 32 + 1


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    o = 0
    W1 = w[o:o + 384].reshape(32, 12); o += 384
    b1 = w[o:o + 32]; o += 32
    W2 = w[o:o + 1024].reshape(32, 32); o += 1024
    b2 = w[o:o + 32]; o += 32
    W3 = w[o:o + 32]; o += 32
    b3 = w[o]
    return W1, b1, W2, b2, W3, b3


def sig(x):
    return 1.0 / (1.0 + np.exp(-x))


def forward(feat, w, amax=0.5):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    x = np.asarray(feat, dtype=np.float64) / 10.0 + 1.0
    p1 = x @ W1.T + b1
    h1 = p1 * sig(p1)
    p2 = h1 @ W2.T + b2
    h2 = p2 * sig(p2)
    z = h2 @ W3 + b3
    return amax * sig(z)


def loss_and_grad(feat, target, w, amax=0.5):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    x = np.asarray(feat, dtype=np.float64) / 10.0 + 1.0
    n = len(x)
    p1 = x @ W1.T + b1
    s1 = sig(p1)
    h1 = p1 * s1
    p2 = h1 @ W2.T + b2
    s2 = sig(p2)
    h2 = p2 * s2
    z = h2 @ W3 + b3
    sz = sig(z)
    out = amax * sz
    r = out - np.asarray(target, dtype=np.float64)
    loss = np.mean(r * r)
    dz = 2.0 * r / n * amax * sz * (1 - sz)
    gW3 = h2.T @ dz
    gb3 = dz.sum()
    d2 = np.outer(dz, W3) * (s2 * (1 + p2 * (1 - s2)))
    gW2 = d2.T @ h1
    gb2 = d2.sum(axis=0)
    d1 = (d2 @ W2) * (s1 * (1 + p1 * (1 - s1)))
    gW1 = d1.T @ x
    gb1 = d1.sum(axis=0)
    grad = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])
    return loss, grad
