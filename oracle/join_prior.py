"""CPU oracle of the learned join-order prior's MLP (test infrastructure:
only tests use it, to check the CUDA forward and backward kernels).

The network is 64 -> 128 -> 128 -> 128 -> 1 with ReLU after each hidden
layer; the loss is mean((y - t)^2).  Parameters are one flat float32 vector
laid out as W1[64][128], b1[128], W2[128][128], b2[128], W3[128][128],
b3[128], w4[128], b4 (W[k][j] maps input k to output j).  Everything here is
float64 numpy, so the GPU's fp32 results are compared against it with a
tolerance.  The reference has no counterpart (its UCT search,
runtime/skinner_join_executor.cc:559-838, uses no learned prior).
"""

import numpy as np

N_IN = 64
N_HID = 128


def unpack(p):
    p = np.asarray(p, np.float64)
    o = 0
    out = {}
    for name, shape in (("W1", (N_IN, N_HID)), ("b1", (N_HID,)), ("W2", (N_HID, N_HID)), ("b2", (N_HID,)),
                        ("W3", (N_HID, N_HID)), ("b3", (N_HID,)), ("w4", (N_HID,)), ("b4", (1,))):
        size = int(np.prod(shape))
        out[name] = p[o:o + size].reshape(shape)
        o += size
    assert o == p.size, (o, p.size)
    return out


def num_params() -> int:
    return N_IN * N_HID + N_HID + 2 * (N_HID * N_HID + N_HID) + N_HID + 1


def forward(p, x):
    w = unpack(p)
    x = np.asarray(x, np.float64)
    h1 = np.maximum(x @ w["W1"] + w["b1"], 0.0)
    h2 = np.maximum(h1 @ w["W2"] + w["b2"], 0.0)
    h3 = np.maximum(h2 @ w["W3"] + w["b3"], 0.0)
    y = h3 @ w["w4"] + w["b4"][0]
    return y, (x, h1, h2, h3)


def gradient(p, x, t):
    """(flat gradient of mean((y - t)^2), loss)."""
    w = unpack(p)
    y, (x, h1, h2, h3) = forward(p, x)
    n = len(y)
    dy = 2.0 * (y - np.asarray(t, np.float64)) / n
    g = {}
    g["w4"] = h3.T @ dy
    g["b4"] = np.array([dy.sum()])
    dz3 = np.outer(dy, w["w4"]) * (h3 > 0)
    g["W3"] = h2.T @ dz3
    g["b3"] = dz3.sum(0)
    dz2 = (dz3 @ w["W3"].T) * (h2 > 0)
    g["W2"] = h1.T @ dz2
    g["b2"] = dz2.sum(0)
    dz1 = (dz2 @ w["W2"].T) * (h1 > 0)
    g["W1"] = x.T @ dz1
    g["b1"] = dz1.sum(0)
    flat = np.concatenate([g[k].ravel() for k in ("W1", "b1", "W2", "b2", "W3", "b3", "w4", "b4")])
    loss = float(np.mean((y - t) ** 2))
    return flat, loss
