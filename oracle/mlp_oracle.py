"""fp64 numpy restatement of the learned lifetime model (test infrastructure).

The MLP 8 -> 64 -> 64 -> 1 with ReLU hidden layers over one flat parameter
array (W1[64][8], b1[64], W2[64][64], b2[64], W3[64], b3), its loss
L = sum_i 0.5 * (MLP(x_i) - t_i)^2 / n and the gradient of L by
back-propagation, all in float64.  The GPU kernels compute the same with
bf16 weights and fp32 accumulation; tests compare them against this at the
same (bf16-representable) weights.  This model has no counterpart in the
reference, which schedules lineages without prediction.
"""
import numpy as np

N_FEATURES = 8
N_HIDDEN = 64
N_PARAMS = 4801
LAYOUT = {"W1": (0, (64, 8)), "b1": (512, (64,)), "W2": (576, (64, 64)),
          "b2": (4672, (64,)), "W3": (4736, (64,)), "b3": (4800, (1,))}


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    return {k: w[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in LAYOUT.items()}


def pack(parts):
    w = np.zeros(N_PARAMS, dtype=np.float64)
    for k, (o, s) in LAYOUT.items():
        w[o:o + int(np.prod(s))] = np.asarray(parts[k], dtype=np.float64).reshape(-1)
    return w


def forward(w, X):
    """MLP(X) for rows of X (n x 8), float64."""
    p = unpack(w)
    X = np.asarray(X, dtype=np.float64)
    h1 = np.maximum(X @ p["W1"].T + p["b1"], 0.0)
    h2 = np.maximum(h1 @ p["W2"].T + p["b2"], 0.0)
    return h2 @ p["W3"] + p["b3"][0]


def loss_and_gradients(w, X, T):
    """(L, dL/dw) for L = sum 0.5 (MLP(x) - t)^2 / n, float64."""
    p = unpack(w)
    X = np.asarray(X, dtype=np.float64)
    T = np.asarray(T, dtype=np.float64)
    n = X.shape[0]
    z1 = X @ p["W1"].T + p["b1"]
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ p["W2"].T + p["b2"]
    h2 = np.maximum(z2, 0.0)
    y = h2 @ p["W3"] + p["b3"][0]
    err = y - T
    L = 0.5 * np.sum(err * err) / n
    dy = err / n
    g = {"W3": h2.T @ dy, "b3": np.array([dy.sum()])}
    d2 = np.outer(dy, p["W3"]) * (z2 > 0)
    g["W2"] = d2.T @ h1
    g["b2"] = d2.sum(axis=0)
    d1 = (d2 @ p["W2"]) * (z1 > 0)
    g["W1"] = d1.T @ X
    g["b1"] = d1.sum(axis=0)
    return L, pack(g)


def to_bf16(w):
    """Round float32 values to the nearest bf16 (ties to even), as float32."""
    a = np.ascontiguousarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    lsb = (a >> 16) & 1
    r = ((a + 0x7FFF + lsb) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32)
