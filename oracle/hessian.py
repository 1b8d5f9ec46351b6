"""Oracle for the ANM Hessian, the half-store Krylov operator, explicit
(Hotelling) deflation and the rigid-body deflation basis.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).  FP64 numpy/scipy.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from . import graph


def hessian_lower(X_nm: np.ndarray, rc_gamma_A: float = 8.0, plus_i: float = 1.0,
                  rowptr=None, cols=None, image=None, box_xy=None):
    """Lower triangle (incl. diagonal) of H + PlusI*I as CSR, and its diagonal.

    Restates InchingLiteInteger/Fuel/T1.py:276-455 without the row batching
    (batching only limits which columns each batch sees; the ungapped columns of
    a batch contain every neighbour of its rows, so the values are the same):
      * x_ij = X_j - X_i (T1.py:276); d2 = xx + yy + zz (T1.py:291);
      * pairs with d2 > rc^2 or d2 == 0 get coefficient 0 (T1.py:292-301);
      * off-diagonal block (i, j) = (x_ij x_ij^T) * (-1/d2) (T1.py:281,307);
      * diagonal block = -sum_j block(i, j), then + PlusI on its three diagonal
        scalars (T1.py:410-421);
      * only scalars on or below the global diagonal are kept (tril, T1.py:444-449)
        and exact zeros are not stored (dense->CSR conversion).
    With periodic xy images (box_xy given; lists from graph.neighbor_lists_pbc_xy
    unless passed with their image codes): the reference's assembly loops over the
    nine instructions for every (i, j) and forms (X_j + box * instr) - X_i
    (Fuel/T1.py:332-334); the neighbour entry found with the query x_i + s is the
    instruction -s, so its pair vector is (X_j - s) - X_i.  Blocks of the same
    (i, j) through different images add up.
    Returns (A_lower csr (3N,3N), A_diag (3N,)).
    """
    X = np.ascontiguousarray(X_nm, dtype=np.float64)
    n = X.shape[0]
    rc = rc_gamma_A / 10.0
    if rowptr is None:
        if box_xy is None:
            _, rowptr, cols = graph.neighbor_lists(X, rc_gamma_A)
        else:
            _, rowptr, cols, image = graph.neighbor_lists_pbc_xy(X, rc_gamma_A, box_xy)
    rows = np.repeat(np.arange(n), np.diff(rowptr))
    if image is None:
        d = X[cols] - X[rows]
    else:
        inst = np.asarray(graph.IMAGES_XY, dtype=np.float64)[np.asarray(image, dtype=np.int64)]
        shift = np.stack([-inst[:, 0] * box_xy[0], -inst[:, 1] * box_xy[1], np.zeros(len(inst))], axis=1)
        d = (X[cols] + shift) - X[rows]
    d2 = d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2]
    mask = (d2 > rc ** 2) | (d2 == 0)
    with np.errstate(divide="ignore"):
        coeff = -1.0 / d2
    coeff[mask] = 0.0
    blocks = d[:, :, None] * d[:, None, :] * coeff[:, None, None]      # (nnzb, 3, 3)
    diag = np.zeros((n, 3, 3))
    np.add.at(diag, rows, -blocks)
    diag[:, [0, 1, 2], [0, 1, 2]] += plus_i
    off = rows != cols if image is None else (rows != cols) | (np.asarray(image) != 0)
    bi = np.concatenate([rows[off], np.arange(n)])
    bj = np.concatenate([cols[off], np.arange(n)])
    bv = np.concatenate([blocks[off], diag])
    p, q = np.meshgrid(np.arange(3), np.arange(3), indexing="ij")
    R = (3 * bi[:, None, None] + p[None]).ravel()
    C = (3 * bj[:, None, None] + q[None]).ravel()
    V = bv.ravel()
    keep = (C <= R) & (V != 0.0)
    A = sp.csr_matrix((V[keep], (R[keep], C[keep])), shape=(3 * n, 3 * n))
    A.sum_duplicates()
    A_diag = A.diagonal().copy()
    return A, A_diag


def full_from_lower(A_lower, A_diag):
    """Symmetric H from its lower triangle: L + L^T - diag."""
    return (A_lower + A_lower.T - sp.diags(A_diag)).tocsr()


def krylov_av(A_lower, A_diag, v):
    """u = [L+D]v + [D+U]v - Dv, InchingLiteInteger/Burn/Krylov/T3.py:128-160."""
    return A_lower @ v + A_lower.T @ v - A_diag * v


def hotelling(Q, x, res, shift):
    """res += shift * Q^T (Q x), Burn/Orthogonalization/T3.py:62-164."""
    return res + shift * (Q.T @ (Q @ x))


def rigid_body_basis(X_nm: np.ndarray) -> np.ndarray:
    """(6, 3N) orthonormal translations + rotations, following the drivers
    (Command8A/commandBenchmark_InchingTRLMHD_Linux_Pdb_0064_A100.py:314-372):
    three unit translations, rotations X @ R_{x,y,z} normalised, then two passes
    of classical Gram-Schmidt applied twice per vector."""
    X = np.asarray(X_nm, dtype=np.float64)
    n = X.shape[0]
    Q = np.zeros((6, 3 * n))
    for i in range(3):
        q = np.zeros((n, 3))
        q[:, i] = 1.0 / np.sqrt(n)
        Q[i] = q.ravel()
    Rx = np.array([[0, 0, 0], [0, 0, -1], [0, 1, 0]], dtype=np.float64).T
    Ry = np.array([[0, 0, 1], [0, 0, 0], [-1, 0, 0]], dtype=np.float64).T
    Rz = np.array([[0, -1, 0], [1, 0, 0], [0, 0, 0]], dtype=np.float64).T
    for t, R in enumerate((Rx, Ry, Rz)):
        g = (X @ R).ravel()
        Q[3 + t] = g / np.linalg.norm(g)
    V = Q.T.copy()
    for _ in range(2):
        for ix in range(1, 6):
            for _twice in range(2):
                V[:, ix] -= V[:, :ix] @ (V[:, :ix].T @ V[:, ix])
                V[:, ix] /= np.sqrt(V[:, ix] @ V[:, ix])
    return V.T.copy()
