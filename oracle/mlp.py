"""CPU oracle of the learned planner's cost model (test infrastructure only:
imported by tests/, never by the library).

The reference has no learned planner; this restates the model the library's
CUDA kernels implement (algo-fft_b200/csrc/gfft_mlp.cu) in float64 numpy, so
the kernels' forward pass and gradients can be checked against it, and its
own gradient against central finite differences.

Model: x (16) -> relu(W1 x + b1) (64) -> relu(W2 h1 + b2) (64) -> w3.h2 + b3.
Flat parameter order: W1[64][16] b1[64] W2[64][64] b2[64] w3[64] b3.
Loss: mean squared error over the samples.
"""
import numpy as np

D, H = 16, 64
NP = H * D + H + H * H + H + H + 1


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + H * D].reshape(H, D); o += H * D
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    w3 = p[o:o + H]; o += H
    b3 = p[o]
    return W1, b1, W2, b2, w3, b3


def forward(p, X):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    X = np.asarray(X, dtype=np.float64).reshape(-1, D)
    a1 = X @ W1.T + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0)
    return h2 @ w3 + b3


def loss_and_grad(p, X, y):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    X = np.asarray(X, dtype=np.float64).reshape(-1, D)
    y = np.asarray(y, dtype=np.float64)
    B = X.shape[0]
    h1 = np.maximum(X @ W1.T + b1, 0)
    h2 = np.maximum(h1 @ W2.T + b2, 0)
    yh = h2 @ w3 + b3
    r = yh - y
    loss = float(np.mean(r * r))
    dy = 2 * r / B
    gw3 = h2.T @ dy
    gb3 = dy.sum()
    d2 = np.outer(dy, w3) * (h2 > 0)
    gW2 = d2.T @ h1
    gb2 = d2.sum(0)
    d1 = (d2 @ W2) * (h1 > 0)
    gW1 = d1.T @ X
    gb1 = d1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gw3, [gb3]])
    return loss, g


def init(seed=0):
    """He-normal weights, zero biases (float32, flat order)."""
    rng = np.random.default_rng(seed)
    W1 = rng.standard_normal((H, D)) * np.sqrt(2.0 / D)
    W2 = rng.standard_normal((H, H)) * np.sqrt(2.0 / H)
    w3 = rng.standard_normal(H) * np.sqrt(1.0 / H)
    return np.concatenate([W1.ravel(), np.zeros(H), W2.ravel(), np.zeros(H), w3, [0.0]]).astype(np.float32)
