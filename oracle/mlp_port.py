"""FP64 NumPy oracle for the learned DSF->Ewald correction (test infrastructure only).

The correction has no counterpart in the reference; this file restates, in plain FP64 NumPy, exactly the
computation the device kernels perform, so their forward values and gradients can be checked:

  descriptors: D[i][32t+k] = sum_{j of species t, r<rc} g_k(r) fc(r),  V[i][32t+k] = sum_j g_k(r) fc(r) d/r
               g_k(r) = exp(-(r - r0 - k dmu)^2 / (2 s^2)),  fc(r) = (cos(pi r / rc) + 1) / 2
  inputs:      X = [(D - mean)/std (64), one-hot species (2), zeros (13), 1]
  network:     H1 = SiLU(X W1^T) (bias = W1[:, 79]); H2 = SiLU(H1 W2^T + b2); C = H2 W3^T + b3
  prediction:  F_i = sum_c C[i, c] V[i, c, :]
  loss:        L = sum_i |F_i - Y_i|^2 / (3 n)
"""
from __future__ import annotations

import numpy as np


def silu(z):
    return z / (1 + np.exp(-z))


def dsilu(z):
    s = 1 / (1 + np.exp(-z))
    return s * (1 + z * (1 - s))


def descriptors(pos, sp, box, rc, r0, dmu, s):
    """Dense O(n^2) restatement of the descriptor kernel (minimum image, FP64)."""
    n = len(pos)
    d = pos[None, :, :] - pos[:, None, :]
    d -= box * np.round(d / box)
    r = np.sqrt(np.einsum("ijk,ijk->ij", d, d))
    np.fill_diagonal(r, np.inf)
    inside = r < rc
    fc = np.where(inside, 0.5 * (np.cos(np.pi * np.where(inside, r, 0) / rc) + 1), 0.0)
    D = np.zeros((n, 64))
    V = np.zeros((n, 64, 3))
    mu = r0 + dmu * np.arange(32)
    rr = np.where(inside, r, 1.0)
    for t in (0, 1):
        mt = inside & (sp[None, :] == t)
        for k in range(32):
            g = np.where(mt, np.exp(-((rr - mu[k]) ** 2) / (2 * s * s)) * fc, 0.0)
            D[:, 32 * t + k] = g.sum(1)
            V[:, 32 * t + k, :] = np.einsum("ij,ijk->ik", g / rr, d)
    return D, V


def inputs(D, sp, mean, inv_std):
    n = len(D)
    X = np.zeros((n, 80))
    X[:, :64] = (D - mean) * inv_std
    X[np.arange(n), 64 + sp] = 1.0
    X[:, 79] = 1.0
    return X


def unpack(theta):
    """Parameter vector [W1 64x80 | W2aug 64x80 | W3aug 64x80] -> W1, W2, b2, W3, b3."""
    t = np.asarray(theta, float).reshape(3, 64, 80)
    return t[0], t[1][:, :64], t[1][:, 64], t[2][:, :64], t[2][:, 64]


def forward(theta, X, V):
    W1, W2, b2, W3, b3 = unpack(theta)
    Z1 = X @ W1.T
    H1 = silu(Z1)
    Z2 = H1 @ W2.T + b2
    H2 = silu(Z2)
    C = H2 @ W3.T + b3
    F = np.einsum("nc,ncd->nd", C, V)
    return F, (Z1, H1, Z2, H2, C)


def loss_and_grad(theta, X, V, Y):
    """Loss and its gradient with respect to the packed parameter vector."""
    W1, W2, b2, W3, b3 = unpack(theta)
    n = len(X)
    F, (Z1, H1, Z2, H2, C) = forward(theta, X, V)
    R = F - Y
    L = float(np.sum(R ** 2) / (3 * n))
    dF = 2 * R / (3 * n)
    dC = np.einsum("nd,ncd->nc", dF, V)
    g = np.zeros((3, 64, 80))
    g[2][:, :64] = dC.T @ H2
    g[2][:, 64] = dC.sum(0)
    dZ2 = (dC @ W3) * dsilu(Z2)
    g[1][:, :64] = dZ2.T @ H1
    g[1][:, 64] = dZ2.sum(0)
    dZ1 = (dZ2 @ W2) * dsilu(Z1)
    g[0] = dZ1.T @ X
    return L, g.reshape(-1), F
