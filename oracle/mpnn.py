"""Oracle of the learned warm start's message-passing network.  TEST
INFRASTRUCTURE ONLY (see oracle/__init__.py).

numpy FP64 restatement of inching_b200.learned.WarmStartMPNN forward/backward
(same layers: node embedding, 3 x [edge-MLP messages averaged per node, node
update with a residual], symmetric edge readout, softplus + floor), plus the
Hellmann-Feynman eigenvalue gradient of a dense bead Hessian.  Used to check
the CUDA kernels' gradients and, by finite differences, itself.
"""
from __future__ import annotations

import numpy as np

FLOOR = 0.05


def relu(x):
    return np.maximum(x, 0.0)


def forward(p, x, ef, src, dst, n_nodes, layers=3):
    """Returns (gamma (E,), cache)."""
    c = {}
    h = relu(x @ p["W0"] + p["b0"])
    c["h0"] = h
    for l in range(layers):
        Z = np.concatenate([h[src], ef], axis=1)
        A = relu(Z @ p[f"Wm{l}"] + p[f"bm{l}"])
        M = np.zeros((n_nodes, A.shape[1]))
        np.add.at(M, dst, A)
        M = M / np.maximum(np.bincount(dst, minlength=n_nodes), 1)[:, None]      # mean over neighbours
        U = np.concatenate([h, M], axis=1)
        T = relu(U @ p[f"Wu{l}"] + p[f"bu{l}"])
        c[l] = (Z, A, U, T)
        h = h + T
    R = np.concatenate([h[dst] + h[src], ef], axis=1)
    s = (R @ p["wo"]).reshape(-1) + p["bo"][0]
    gamma = np.logaddexp(0.0, s) + FLOOR
    c["R"], c["s"] = R, s
    return gamma, c


def backward(p, x, ef, src, dst, n_nodes, c, dgamma, layers=3):
    g = {k: np.zeros_like(v) for k, v in p.items()}
    ds = dgamma / (1.0 + np.exp(-c["s"]))
    g["wo"] = c["R"].T @ ds[:, None]
    g["bo"] = np.array([ds.sum()])
    dR = ds[:, None] * p["wo"].reshape(1, -1)
    W = p["W0"].shape[1]
    dh = np.zeros((n_nodes, W))
    np.add.at(dh, dst, dR[:, :W])
    np.add.at(dh, src, dR[:, :W])
    for l in reversed(range(layers)):
        Z, A, U, T = c[l]
        dT = dh * (T > 0)
        g[f"Wu{l}"] = U.T @ dT
        g[f"bu{l}"] = dT.sum(axis=0)
        dU = dT @ p[f"Wu{l}"].T
        dM = dU[:, W:] / np.maximum(np.bincount(dst, minlength=n_nodes), 1)[:, None]
        dh = dh + dU[:, :W]
        dA = dM[dst] * (A > 0)
        g[f"Wm{l}"] = Z.T @ dA
        g[f"bm{l}"] = dA.sum(axis=0)
        dZ = dA @ p[f"Wm{l}"].T
        np.add.at(dh, src, dZ[:, :W])
    dh = dh * (c["h0"] > 0)
    g["W0"] = x.T @ dh
    g["b0"] = dh.sum(axis=0)
    return g


def bead_hessian(pos, src, dst, gamma, plus_i=1.0):
    """Dense Hessian of a spring network: pair (a, b) with constant gamma_e (each
    direction carries the pair's constant) -> blocks -gamma u u^T, diagonal sums."""
    n = pos.shape[0]
    H = np.zeros((3 * n, 3 * n))
    for e in range(len(src)):
        a, b = dst[e], src[e]
        u = pos[b] - pos[a]
        u = u / np.linalg.norm(u)
        B = gamma[e] * np.outer(u, u)
        H[3 * a:3 * a + 3, 3 * b:3 * b + 3] -= B
        H[3 * a:3 * a + 3, 3 * a:3 * a + 3] += B
    return H + plus_i * np.eye(3 * n)


def hf_grad(pos, src, dst, V, c):
    """out[e] = 1/2 sum_t c_t (u_e . (V_t[a] - V_t[b]))^2."""
    out = np.zeros(len(src))
    for e in range(len(src)):
        a, b = dst[e], src[e]
        u = pos[b] - pos[a]
        u = u / np.linalg.norm(u)
        d = V[3 * a:3 * a + 3] - V[3 * b:3 * b + 3]
        out[e] = 0.5 * np.sum(c * (u @ d) ** 2)
    return out
