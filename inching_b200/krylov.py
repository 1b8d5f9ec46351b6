"""Operators on the Hessian store: H v (+ explicit deflation) and the Chebyshev
filter p(H) v, both built on the fused SpMM kernel.

Reference counterparts:
  * KrylovAv factories  -- InchingLiteInteger/Burn/Krylov/T3.py:54-239
  * Hotelling update    -- Burn/Orthogonalization/T3.py:62-164 (res += s Q^T Q x)
  * ChebyshevAv         -- Burn/PolynomialFilters/T2.py:16-92 (three-term recurrence
                           y = sum_k mu_k T_k((H - cc)/dd) v, KPM density term)
"""
from __future__ import annotations

import math

import torch


def _vec_dtype(prec):
    return torch.float64 if prec == 64 else torch.float32


class HessianOperator:
    """u = H v [+ shift * Q^T Q v] in the requested store precision.

    Vectors are FP64 at the interface; with prec=32 the product runs on the FP32
    store with FP32 vectors (inputs rounded once, output widened once)."""

    def __init__(self, A, prec=64, Q=None, hot_shift=0.0):
        self.A = A
        self.prec = prec
        self.Q = None if Q is None else _as_dense_q(Q, A)
        self.hot_shift = float(hot_shift)
        self.n = A.shape[0]

    def __call__(self, v, out=None, alpha=1.0, gamma=0.0, deflate=True):
        Q = self.Q if deflate else None
        kw = dict(alpha=alpha, gamma=gamma, Q=Q, hot_shift=self.hot_shift if Q is not None else 0.0)
        if self.prec == 64:
            if out is None:
                out = torch.empty_like(v)
            return self.A.matmul(v.contiguous(), out=out, prec=64, **kw)
        v32 = v.to(torch.float32).contiguous()
        y32 = self.A.matmul(v32, prec=32, **kw)
        if out is None:
            return y32.to(torch.float64)
        out.copy_(y32)
        return out


def _as_dense_q(Q, A):
    """Deflation basis as a dense (r, 3N) FP64 CUDA tensor.  Accepts torch, numpy
    or scipy sparse (the reference passes a CSR-ified dense Q)."""
    if isinstance(Q, torch.Tensor):
        q = Q
    else:
        try:
            import scipy.sparse as sp
            if sp.issparse(Q):
                Q = Q.toarray()
        except ImportError:  # pragma: no cover
            pass
        import numpy as np
        q = torch.from_numpy(np.asarray(Q, dtype=np.float64))
    q = q.to(device=A.device, dtype=torch.float64).contiguous()
    if q.dim() != 2 or q.shape[1] != A.shape[0]:
        raise AssertionError("ABORTED. the Hotelling basis must have shape (r, n)")
    if q.shape[0] > 8:
        raise AssertionError("ABORTED. at most 8 Hotelling deflation vectors are fused into the operator")
    return q


class ChebyshevFilter:
    """y = sum_{k=0..m} mu_k T_k((H - cc)/dd) v, one fused SpMM per degree:
    X_{k+1} = (s/dd)(H X_k - cc X_k) - X_{k-1}  (s = 1 for k = 1, else 2) and
    Y += mu_{k+1} X_{k+1} in the same kernel.  Works on (n,) or (n, b) blocks."""

    def __init__(self, A, params, prec=64):
        self.A = A
        self.p = params
        self.prec = prec

    @property
    def degree(self):
        return int(self.p.AdjustedDegree)

    def __call__(self, v, return_rho=False):
        p = self.p
        mu = [float(x) for x in p.AdjustedCoefficients]
        m = int(p.AdjustedDegree)
        cc, dd = float(p.cc), float(p.dd)
        dt = _vec_dtype(self.prec)
        x0 = v.to(dt).contiguous()
        y = x0 * mu[0]
        if m == 0:
            return y.to(v.dtype)
        vkm1 = torch.empty_like(x0)
        vk = x0.clone()
        rho = None
        if return_rho:
            jac = p.AdjustedDampingKernels
            rho = p.theta_a - p.theta_b
            ta, tb = p.theta_a, p.theta_b
        for k in range(1, m + 1):
            scal = 1.0 / dd if k == 1 else 2.0 / dd
            if k == 1:
                self.A.matmul(vk, out=vkm1, prec=self.prec, alpha=scal, gamma=-scal * cc, acc=y, mu=mu[k])
            else:
                self.A.matmul(vk, out=vkm1, prec=self.prec, alpha=scal, gamma=-scal * cc, beta=-1.0, Yin=vkm1,
                              acc=y, mu=mu[k])
            vk, vkm1 = vkm1, vk
            if return_rho:
                rho = rho - 2 * float(jac[k]) * torch.dot(vk.double().flatten(), v.double().flatten()) * (
                    math.sin(k * tb) - math.sin(k * ta)) / k
        out = y.to(v.dtype)
        if return_rho:
            return out, rho / math.pi
        return out
