"""CPU oracle of the configuration predictor's network (test infrastructure:
only tests/ use it).

The reference has no learned predictor (its configuration choice is a static
table lookup, src/hml_sgemm_kernel.cu:189-237), so this is a restatement of
the library's own network in numpy float64, the checker for the GPU training
and inference kernels (hiperml_b200/csrc/predictor.cu):

    h1 = relu(W1 f + b1), h2 = relu(W2 h1 + b2), s = W3 h2 + b3
    loss = sum_{i,j} w_ij (s_ij - y_ij)^2 / sum w

It is pinned by central finite differences of its own loss
(tests/test_predictor.py), not by reference outputs: parity with the
reference is not applicable to this part.
"""
import numpy as np

N_IN, N_HID = 5, 64


def split(params, C):
    p = np.asarray(params, np.float64)
    o = 0
    out = {}
    for name, shape in (("W1", (N_HID, N_IN)), ("b1", (N_HID,)), ("W2", (N_HID, N_HID)),
                        ("b2", (N_HID,)), ("W3", (C, N_HID)), ("b3", (C,))):
        n = int(np.prod(shape))
        out[name] = p[o:o + n].reshape(shape)
        o += n
    assert o == len(p), (o, len(p))
    return out


def forward(params, C, X):
    P = split(params, C)
    X = np.asarray(X, np.float64)
    z1 = X @ P["W1"].T + P["b1"]
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ P["W2"].T + P["b2"]
    h2 = np.maximum(z2, 0.0)
    s = h2 @ P["W3"].T + P["b3"]
    return s, (X, z1, h1, z2, h2)


def loss(params, C, X, Y, W):
    s, _ = forward(params, C, X)
    W = np.asarray(W, np.float64)
    return float((W * (s - np.asarray(Y, np.float64)) ** 2).sum() / W.sum())


def loss_grad(params, C, X, Y, W):
    """Analytic loss and gradient (same layout as params)."""
    P = split(params, C)
    s, (X, z1, h1, z2, h2) = forward(params, C, X)
    W = np.asarray(W, np.float64)
    d = s - np.asarray(Y, np.float64)
    L = float((W * d * d).sum() / W.sum())
    ds = 2.0 * W * d / W.sum()
    gW3 = ds.T @ h2
    gb3 = ds.sum(0)
    dh2 = ds @ P["W3"] * (z2 > 0)
    gW2 = dh2.T @ h1
    gb2 = dh2.sum(0)
    dh1 = dh2 @ P["W2"] * (z1 > 0)
    gW1 = dh1.T @ X
    gb1 = dh1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return L, g


def predict(params, C, X, allow):
    """argmin of the scores over allowed configurations (lowest index on
    ties, -1 when none is allowed), and the scores."""
    s, _ = forward(params, C, X)
    masked = np.where(np.asarray(allow, bool), s, np.inf)
    idx = np.argmin(masked, axis=1)
    idx = np.where(np.isinf(masked[np.arange(len(idx)), idx]), -1, idx)
    return idx, s


def features(M, N, K, akc, bkc):
    """The predictor's features of a canonical (long-M) problem."""
    return np.array([np.log2(max(1, M)) / 16.0, np.log2(max(1, N)) / 8.0,
                     np.log2(max(1, K)) / 14.0, float(akc), float(bkc)])
