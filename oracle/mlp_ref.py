"""NumPy restatement of the cost model's network.  TEST INFRASTRUCTURE.

The checker for the library's CUDA forward / backward kernels
(flint_b200/csrc/mlp_kernels.cuh): the same parameter layout
W1[n_in][64], b1[64], W2[64][64], b2[64], W3[64][64], b3[64], W4[64], b4,
ReLU hidden layers, mean squared error (1/n) sum (y - t)^2, computed in float64.
The reference has no learned component; this oracle is pinned by central
finite differences of its own loss (tests/test_oracle.py).
"""
import numpy as np

H = 64


def offsets(n_in):
    o = {}
    k = 0
    for name, size in (("W1", n_in * H), ("b1", H), ("W2", H * H), ("b2", H), ("W3", H * H),
                       ("b3", H), ("W4", H), ("b4", 1)):
        o[name] = (k, size)
        k += size
    o["total"] = k
    return o


def unpack(P, n_in):
    o = offsets(n_in)
    P = np.asarray(P, dtype=np.float64)
    g = {name: P[v[0]:v[0] + v[1]] for name, v in o.items() if name != "total"}
    return (g["W1"].reshape(n_in, H), g["b1"], g["W2"].reshape(H, H), g["b2"],
            g["W3"].reshape(H, H), g["b3"], g["W4"], g["b4"][0])


def forward(P, X):
    X = np.asarray(X, dtype=np.float64)
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(P, X.shape[1])
    z1 = X @ W1 + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2 + b2
    h2 = np.maximum(z2, 0)
    z3 = h2 @ W3 + b3
    h3 = np.maximum(z3, 0)
    y = h3 @ W4 + b4
    return y, (h1, h2, h3)


def loss(P, X, t):
    y, _ = forward(P, X)
    return float(np.mean((y - np.asarray(t, dtype=np.float64)) ** 2))


def gradient(P, X, t):
    """Gradient of the mean squared error with respect to the parameter vector."""
    X = np.asarray(X, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    n, n_in = X.shape
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(P, n_in)
    y, (h1, h2, h3) = forward(P, X)
    dy = 2.0 * (y - t) / n
    gW4 = h3.T @ dy
    gb4 = dy.sum()
    d3 = np.outer(dy, W4) * (h3 > 0)
    gW3 = h2.T @ d3
    gb3 = d3.sum(0)
    d2 = (d3 @ W3.T) * (h2 > 0)
    gW2 = h1.T @ d2
    gb2 = d2.sum(0)
    d1 = (d2 @ W2.T) * (h1 > 0)
    gW1 = X.T @ d1
    gb1 = d1.sum(0)
    return np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3, gW4, [gb4]])
