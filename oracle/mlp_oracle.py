"""FP64 numpy statement of the smoothing-length MLP's forward and backward
pass (12 -> 64 -> 64 -> 1, SiLU, mean-squared loss).

TEST INFRASTRUCTURE ONLY: the checker for the library's tensor-core kernels.
The network has no counterpart in the reference.  To compare like with like,
the values the GPU rounds to BF16 before a tensor-core product (inputs, W1,
W2, the first-layer activations and the two hidden-layer deltas) are rounded
the same way here; everything else is FP64.
"""
import numpy as np

N_IN, N_INP, N_H = 12, 16, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + N_H * N_INP
OFF_W2 = OFF_B1 + N_H
OFF_B2 = OFF_W2 + N_H * N_H
OFF_W3 = OFF_B2 + N_H
OFF_B3 = OFF_W3 + N_H
N_PARAM = OFF_B3 + 1


def bf16(a):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    rounding = ((u >> 16) & 1) + 0x7FFF
    u = ((u + rounding) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    W1 = p[OFF_W1:OFF_B1].reshape(N_H, N_INP)
    b1 = p[OFF_B1:OFF_W2]
    W2 = p[OFF_W2:OFF_B2].reshape(N_H, N_H)
    b2 = p[OFF_B2:OFF_W3]
    w3 = p[OFF_W3:OFF_B3]
    b3 = p[OFF_B3]
    return W1, b1, W2, b2, w3, b3


def silu(x):
    return x / (1.0 + np.exp(-x))


def dsilu(x):
    s = 1.0 / (1.0 + np.exp(-x))
    return s * (1.0 + x * (1.0 - s))


def forward_backward(params, X, y):
    """Returns (out, loss, grad) for raw features X (rows x 12) and targets y."""
    W1, b1, W2, b2, w3, b3 = unpack(params)
    rows = X.shape[0]
    Xp = np.zeros((rows, N_INP))
    Xp[:, :N_IN] = X
    Xb = bf16(Xp)
    W1b, W2b = bf16(W1), bf16(W2)
    H1 = Xb @ W1b.T + b1
    A1b = bf16(silu(H1))
    H2 = A1b @ W2b.T + b2
    A2 = silu(H2)
    out = A2 @ w3 + b3
    diff = out - y
    loss = np.sum(diff * diff) / rows
    dout = 2.0 * diff / rows
    dw3 = A2.T @ dout
    db3 = dout.sum()
    dH2 = dout[:, None] * w3[None, :] * dsilu(H2)
    db2 = dH2.sum(0)
    dH2b = bf16(dH2)
    dA1 = dH2b @ W2b
    dH1 = dA1 * dsilu(H1)
    db1 = dH1.sum(0)
    dW2 = dH2b.T @ A1b
    dW1 = bf16(dH1).T @ Xb
    dW1[:, N_IN:] = 0.0
    g = np.zeros(N_PARAM)
    g[OFF_W1:OFF_B1] = dW1.ravel()
    g[OFF_B1:OFF_W2] = db1
    g[OFF_W2:OFF_B2] = dW2.ravel()
    g[OFF_B2:OFF_W3] = db2
    g[OFF_W3:OFF_B3] = dw3
    g[OFF_B3] = db3
    return out, loss, g


def numeric_grad(params, X, y, idx, eps=1e-6):
    """Central differences of the loss of the unrounded FP64 network (sanity
    check of the analytic backward pass itself)."""
    def loss_of(p):
        W1, b1, W2, b2, w3, b3 = unpack(p)
        Xp = np.zeros((X.shape[0], N_INP))
        Xp[:, :N_IN] = X
        out = silu(silu(Xp @ W1.T + b1) @ W2.T + b2) @ w3 + b3
        return np.mean((out - y) ** 2)
    g = []
    for i in idx:
        p1 = np.array(params, dtype=np.float64)
        p2 = p1.copy()
        p1[i] += eps
        p2[i] -= eps
        g.append((loss_of(p1) - loss_of(p2)) / (2 * eps))
    return np.array(g)
