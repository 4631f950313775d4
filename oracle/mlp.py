"""Test infrastructure (the oracle): a NumPy restatement, in FP64, of the
selector network's forward and backward passes (opt_solver_b200/csrc/
smfg_mlp.cu), the checker of the CUDA kernels' gradients. Parameters packed
as W1 (h x d), b1 (h), w2 (h), b2 (1); loss = sum_s w_s BCE(p_s, y_s) / n."""
import numpy as np


def unpack(P, d, h):
    P = np.asarray(P, dtype=np.float64)
    W1 = P[:h * d].reshape(h, d)
    b1 = P[h * d:h * d + h]
    w2 = P[h * d + h:h * d + 2 * h]
    b2 = P[h * d + 2 * h]
    return W1, b1, w2, b2


def forward(P, X, d, h):
    W1, b1, w2, b2 = unpack(P, d, h)
    Z1 = X @ W1.T + b1
    A = np.maximum(Z1, 0.0)
    z2 = A @ w2 + b2
    return 1.0 / (1.0 + np.exp(-z2)), Z1, A


def loss_and_grad(P, X, y, w, d, h):
    X = np.asarray(X, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    n = X.shape[0]
    w = np.ones(n) if w is None else np.asarray(w, dtype=np.float64)
    p, Z1, A = forward(P, X, d, h)
    pc = np.clip(p, 1e-7, 1 - 1e-7)
    loss = float(np.sum(-w * (y * np.log(pc) + (1 - y) * np.log(1 - pc))) / n)
    W1, b1, w2, b2 = unpack(P, d, h)
    dz2 = w * (p - y) / n
    dw2 = A.T @ dz2
    db2 = dz2.sum()
    dZ1 = np.outer(dz2, w2) * (Z1 > 0)
    dW1 = dZ1.T @ X
    db1 = dZ1.sum(axis=0)
    return loss, np.concatenate([dW1.reshape(-1), db1, dw2, [db2]])
