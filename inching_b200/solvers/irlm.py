"""Implicitly restarted Lanczos with explicit (Hotelling) deflation, on the GPU.

Follows InchingLiteInteger/Burn/ImplicitlyRestartedLanczosHotellingDeflation/T1.py
(and its description in Tex/main.tex:259-318):
  * p = min(max(2k, k+32), n-1), two extra kept Ritz vectors (k += 2)     (T1.py:345-351)
  * p-step Lanczos extension with random restart on breakdown and two passes
    of Gram-Schmidt against all earlier vectors but the previous one     (T1.py:85-215)
  * p exact shifts = the p largest Ritz values, one QR per shift on the
    (k+p) tridiagonal, basis compressed to k vectors                     (T1.py:231-298)
  * convergence by the Paige bound |beta[k-2]| < tol                      (T1.py:66-77,445)
  * final tridiagonal eigensolve and rotation of the kept basis           (T1.py:452-477)
The reference builds its operator with one argument (T1.py:368), which the
operator factory rejects; here the operator is the store's own SpMM (H v with
the fused Hotelling term).  The small tridiagonal/QR work runs on the host
(LAPACK); vectors and Gram-Schmidt stay on the GPU in FP64.
"""
from __future__ import annotations

import numpy as np
import torch

from ..krylov import HessianOperator


def _orth_all_before(V, ix, before):
    """V[ix] -= V[:before]^T (V[:before] V[ix]); normalise (Orthogonalization/T1.py:56-64)."""
    if before > 0:
        B = V[:before]
        V[ix] -= B.t().mv(B.mv(V[ix]))
    V[ix] /= torch.linalg.vector_norm(V[ix])


def _lanczos_ext(op, a, b, V, k, p, tol, gen):
    n = V.shape[1]
    for j in range(p):
        idx = k + j - 1
        if idx == 0 or abs(b[idx - 1]) < tol:
            V[idx] = torch.rand(n, generator=gen, dtype=torch.float64, device=V.device)
            if idx > 1:
                _orth_all_before(V, idx, idx - 1)
                _orth_all_before(V, idx, idx - 1)
            else:
                V[idx] /= torch.linalg.vector_norm(V[idx])
        u = op(V[idx])
        if idx > 0:
            h = V[idx - 1:idx + 1].mv(u)
            hh = h.cpu().numpy()
            a[idx] = hh[1]
            b[idx] = hh[0]
            V[idx + 1] = u - V[idx - 1:idx + 1].t().mv(h)
        else:
            h = float(torch.dot(V[0], u))
            a[0] = h
            V[1] = u - V[0] * h
        beta = float(torch.linalg.vector_norm(V[idx + 1]))
        if beta > tol:
            V[idx + 1] /= beta
            b[idx] = beta
        else:
            b[idx] = 0.0
            continue
        _orth_all_before(V, idx + 1, idx)
        _orth_all_before(V, idx + 1, idx)


def _tridiag(a, b):
    return np.diag(a) + np.diag(b, 1) + np.diag(b, -1)


def _implicit_shift(V, a, b, k, p):
    T = _tridiag(a, b[:k + p - 1])
    ev = np.linalg.eigvalsh(T)
    shifts = np.argsort(ev)[::-1][:p]
    Qacc = np.eye(k + p)
    for i in shifts:
        T = _tridiag(a, b[:k + p - 1])
        lastb = b[k + p - 1:k + p].copy()
        Qj = np.linalg.qr(T - ev[i] * np.eye(k + p), mode="complete")[0]
        T = Qj.T @ (T @ Qj)
        a = np.diagonal(T).copy()
        b = np.concatenate((np.diagonal(T, 1), lastb))
        Qacc = Qacc @ Qj
    Qt = torch.from_numpy(np.ascontiguousarray(Qacc.T)).to(V.device)
    v = Qt[k] @ V[:k + p]
    V[:k] = Qt[:k] @ V[:k + p]
    V[k] = b[k - 1] * v + (b[k + p - 1] * float(Qacc.T[k - 1, k + p - 1])) * V[k + p]
    beta = float(torch.linalg.vector_norm(V[k]))
    V[k] /= beta
    b[k - 1] = beta
    _orth_all_before(V, k, k)
    _orth_all_before(V, k, k)
    return a, b


def irlm(A, k=32, maxiter=15000, tol=1e-8, Q=None, shift=10.0, precision="f64", seed=0, return_info=False):
    n = A.shape[0]
    assert k < n, "ABORTED. k must be smaller than n"
    assert A.ndim == 2, "ABORTED. It is a tensor not rank 2!"
    assert A.shape[0] == A.shape[1], "ABORTED. square"
    assert k >= 32, "ABORTED. we did not test on less than 32 modes, as the number ritz vectors is too small."
    p = min(max(2 * k, k + 32), n - 1)
    k += 2
    m = k + p
    assert n >= m, "ABORTED. You sure you want more basis than number of columns of A?"
    if tol == 0:
        tol = float(np.finfo(np.float64).eps)
    dev = A.device
    op = HessianOperator(A, prec=32 if precision == "mixed" else 64, Q=Q, hot_shift=shift)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    V = torch.zeros((m + 1, n), dtype=torch.float64, device=dev)
    a = np.zeros(m)
    b = np.zeros(m)
    _lanczos_ext(op, a, b, V, 1, k, tol, gen)
    it = 0
    converged = False
    for it in range(maxiter):
        _lanczos_ext(op, a, b, V, k + 1, p, tol, gen)
        a, b = _implicit_shift(V, a, b, k, p)
        if abs(b[k - 1]) < tol:
            b[k - 1] = 0.0
        if abs(b[k]) < tol:
            b[k] = 0.0
        if abs(b[k - 2]) < tol:
            converged = True
            break
    T = _tridiag(a[:k], b[:k - 1])
    tval, tvec = np.linalg.eigh(T, UPLO="L")
    W = torch.from_numpy(np.ascontiguousarray(tvec[:k - 1, :k - 1].T)).to(dev)
    V[:k - 1] = W @ V[:k - 1]
    evals = torch.from_numpy(tval[:k - 2].copy()).to(dev)
    evecs = V[:k - 2].t().contiguous()
    if return_info:
        return evals, evecs, dict(iterations=it + 1, converged=converged, paige_bound=abs(b[k - 2]))
    return evals, evecs
