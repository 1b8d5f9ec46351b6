"""Thick-restart Lanczos with explicit (Hotelling) deflation and optional
Chebyshev filtering, on the GPU.

Follows InchingLiteInteger/Burn/ThickRestartLanczosHotellingDeflation/T1.py:
  * workspace ncv = min(max(f*k, k+32), n-1), tol = eps if 0          (T1.py:94-98)
  * p-step Lanczos with two full reorthogonalisation passes per step  (T1.py:436-520)
  * tridiagonal / arrowhead Rayleigh-Ritz on the host (LAPACK), k smallest
    (k largest of p(H) when a polynomial filter is used)             (T1.py:320-351)
  * thick restart V[:k] = W^T V, residual ||beta_k|| <= tol            (T1.py:176-260)
  * under a filter, eigenvalues recovered as Rayleigh quotients        (T1.py:277-291)
The operator is the fused SpMM (H v + shift Q^T Q v in one kernel) on the FP64
store, or on the FP32 store when precision="mixed" (Lanczos vectors, projections
and Ritz values stay FP64).
"""
from __future__ import annotations

import numpy as np
import torch

from ..krylov import ChebyshevFilter, HessianOperator


def _tridiag_eig(alpha, beta, beta_k, k, filtered):
    a = alpha.cpu().numpy()
    b = beta.cpu().numpy()
    t = np.diag(a) + np.diag(b[:-1], 1) + np.diag(b[:-1], -1)
    if beta_k is not None:
        bk = beta_k.cpu().numpy()
        t[k, :k] = bk
        t[:k, k] = bk
    S, W = np.linalg.eigh(t)
    idx = np.argsort(S)
    sel = idx[-k:][::-1] if filtered else idx[:k]
    return S[sel], W[:, sel]


class _Apply:
    def __init__(self, A, precision, Q, shift, polynomial):
        prec = 32 if precision == "mixed" else 64
        self.op = HessianOperator(A, prec=prec, Q=Q, hot_shift=shift)
        self.cheb = None if polynomial is None else ChebyshevFilter(A, polynomial, prec=prec)
        self.plain = HessianOperator(A, prec=prec)
        self.n_spmm = 0

    def __call__(self, v, out):
        if self.cheb is None:
            self.n_spmm += 1
            return self.op(v, out=out)
        self.n_spmm += self.cheb.degree
        y = self.cheb(v)
        if self.op.Q is not None:
            Q = self.op.Q
            y = y + self.op.hot_shift * (Q.T @ (Q @ v))
        out.copy_(y)
        return out


def _lanczos(apply, V, u, alpha, beta, i_start, i_end):
    v = V[i_start].clone()
    for i in range(i_start, i_end):
        apply(v, u)
        alpha[i] = torch.dot(v, u)
        Vi = V[:i + 1]
        u.sub_(Vi.t().mv(Vi.mv(u)))
        beta[i] = torch.linalg.vector_norm(u)
        u.sub_(Vi.t().mv(Vi.mv(u)))
        if i >= i_end - 1:
            break
        torch.div(u, beta[i], out=v)
        V[i + 1] = v


def trlm(A, k=32, maxiter=10000, tol=0.0, workspace_factor=2, Q=None, shift=10.0, polynomial=None,
         precision="f64", seed=0, return_info=False):
    """k lowest eigenpairs of the store A (eigenvalues ascending, incl. PlusI)."""
    N = A.shape[0]
    assert k < N, "ABORTED. k must be smaller than n"
    assert A.ndim == 2, "ABORTED. It is a tensor not rank 2!"
    assert A.shape[0] == A.shape[1], "ABORTED. square"
    assert precision in ("f64", "mixed"), "ABORTED. precision must be 'f64' or 'mixed'"
    dev = A.device
    ncv = min(max(workspace_factor * k, k + 32), N - 1)
    if tol == 0:
        tol = float(np.finfo(np.float64).eps)
    apply = _Apply(A, precision, Q, shift, polynomial)
    filtered = polynomial is not None
    f64 = torch.float64
    alpha = torch.zeros(ncv, dtype=f64, device=dev)
    beta = torch.zeros(ncv, dtype=f64, device=dev)
    V = torch.empty((ncv, N), dtype=f64, device=dev)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    u = torch.rand(N, generator=g, dtype=f64, device=dev)
    V[0] = u / torch.linalg.vector_norm(u)

    _lanczos(apply, V, u, alpha, beta, 0, ncv)
    S, W = _tridiag_eig(alpha, beta, None, k, filtered)
    Wd = torch.from_numpy(np.ascontiguousarray(W)).to(dev)
    V[:k] = Wd.t() @ V
    beta_k = beta[-1] * Wd[-1, :]
    res = float(torch.linalg.vector_norm(beta_k))
    it = 0
    for it in range(maxiter):
        beta[:k] = 0
        alpha[:k] = torch.from_numpy(S).to(dev)
        u.sub_(V[:k].t().mv(V[:k].mv(u)))
        u.div_(torch.linalg.vector_norm(u))
        V[k] = u
        apply(V[k], u)
        alpha[k] = torch.dot(V[k], u)
        u.sub_(alpha[k] * V[k])
        u.sub_(V[:k].t().mv(beta_k))
        beta[k] = torch.linalg.vector_norm(u)
        V[k + 1] = u / beta[k]
        _lanczos(apply, V, u, alpha, beta, k + 1, ncv)
        S, W = _tridiag_eig(alpha, beta, beta_k, k, filtered)
        Wd = torch.from_numpy(np.ascontiguousarray(W)).to(dev)
        V[:k] = Wd.t() @ V
        beta_k = beta[-1] * Wd[-1, :]
        res = float(torch.linalg.vector_norm(beta_k))
        if res <= tol:
            break
    Vk = V[:k]
    if filtered:
        plain = HessianOperator(A, prec=64)
        HV = plain(Vk.t().contiguous())
        S = (Vk.t() * HV).sum(dim=0).cpu().numpy()
    else:
        S = np.asarray(S)
    idx = np.argsort(S)
    idx_t = torch.from_numpy(idx).to(dev)
    evals = torch.from_numpy(S[idx].copy()).to(dev)
    evecs = Vk[idx_t].t().contiguous()
    if return_info:
        return evals, evecs, dict(iterations=it + 1, residual=res, n_spmm=apply.n_spmm, ncv=ncv,
                                  converged=res <= tol)
    return evals, evecs
