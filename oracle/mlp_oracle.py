"""ORACLE — test infrastructure only.

numpy restatement of the learned style selector's network and loss, used to
check the engine's hand-written CUDA forward/backward kernels
(indigo2suite_b200/csrc/selector.cu) and its on-device inference.

Parameter blob layout (float32), identical to the engine's:
  mu[16], sd[16]                     input standardisation (not trained)
  W1[16][64], b1[64]                 weights stored [in][out]
  W2[64][64], b2[64]
  W3[64][9],  b3[9]                  one output per variant
Forward: x_s = (x - mu) / sd; h1 = relu(x_s W1 + b1); h2 = relu(h1 W2 + b2);
y = h2 W3 + b3 (predicted log2 launch time per variant).
Loss: sum(M * (y - T)^2) / sum(M).
"""
from __future__ import annotations

import numpy as np

F, H, O = 16, 64, 9
OFF_MU = 0
OFF_SD = OFF_MU + F
OFF_W1 = OFF_SD + F
OFF_B1 = OFF_W1 + F * H
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H * O
NPARAMS = OFF_B3 + O


def unpack(p: np.ndarray):
    p = np.asarray(p, np.float64)
    return (p[OFF_MU:OFF_SD], p[OFF_SD:OFF_W1], p[OFF_W1:OFF_B1].reshape(F, H), p[OFF_B1:OFF_W2],
            p[OFF_W2:OFF_B2].reshape(H, H), p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3].reshape(H, O), p[OFF_B3:NPARAMS])


def init_params(seed: int = 0) -> np.ndarray:
    """He-initialised weights, zero biases, identity standardisation."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAMS, np.float32)
    p[OFF_SD:OFF_W1] = 1.0
    p[OFF_W1:OFF_B1] = rng.normal(0, np.sqrt(2.0 / F), F * H)
    p[OFF_W2:OFF_B2] = rng.normal(0, np.sqrt(2.0 / H), H * H)
    p[OFF_W3:OFF_B3] = rng.normal(0, np.sqrt(1.0 / H), H * O)
    return p


def forward(p, X):
    mu, sd, W1, b1, W2, b2, W3, b3 = unpack(p)
    xs = (np.asarray(X, np.float64) - mu) / sd
    z1 = xs @ W1 + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2 + b2
    h2 = np.maximum(z2, 0)
    y = h2 @ W3 + b3
    return xs, z1, h1, z2, h2, y


def loss_grad(p, X, T, M):
    """Loss and its gradient w.r.t. every parameter (normaliser gradient = 0)."""
    mu, sd, W1, b1, W2, b2, W3, b3 = unpack(p)
    xs, z1, h1, z2, h2, y = forward(p, X)
    M = np.asarray(M, np.float64)
    cnt = M.sum()
    diff = y - np.asarray(T, np.float64)
    loss = float((M * diff * diff).sum() / cnt)
    dy = 2.0 * M * diff / cnt
    g = np.zeros(NPARAMS, np.float64)
    g[OFF_W3:OFF_B3] = (h2.T @ dy).ravel()
    g[OFF_B3:NPARAMS] = dy.sum(0)
    d2 = (dy @ W3.T) * (z2 > 0)
    g[OFF_W2:OFF_B2] = (h1.T @ d2).ravel()
    g[OFF_B2:OFF_W3] = d2.sum(0)
    d1 = (d2 @ W2.T) * (z1 > 0)
    g[OFF_W1:OFF_B1] = (xs.T @ d1).ravel()
    g[OFF_B1:OFF_W2] = d1.sum(0)
    return loss, g


def predict(p, X, allowed_mask: int = (1 << O) - 1) -> np.ndarray:
    y = forward(p, X)[-1]
    allowed = np.array([(allowed_mask >> k) & 1 for k in range(O)], bool)
    y = np.where(allowed[None, :], y, np.inf)
    return np.argmin(y, axis=1).astype(np.int32)
