"""Jacobi-Davidson with explicit (Hotelling) deflation, on the GPU.

Follows InchingLiteInteger/Burn/JacobiDavidsonHotellingDeflation/T1.py:382-757:
  * search space V (jmax = f*k), locked Ritz vectors Q, projected matrix G;
    G's eigenproblem is solved on the host (LAPACK, UPLO='L')        (T1.py:534-541)
  * smallest Ritz pair, residual r = H u - theta u; converged pairs are locked and
    removed from the search space                                     (T1.py:543-657)
  * restart to jmin = k Ritz vectors when V is full                  (T1.py:662-666)
  * correction (I - uu^T)(H - sigma I)(I - uu^T) z = -r by projected GMRES(20),
    sigma = theta if ||r|| < 1e-3 else theta - gap, tolerance ||r||*1e-4
    (T1.py:669-698, IterativeSolvers.py:216-305, including its return of the
    projected iterate and its output projection with (uu . z))
  * z orthogonalised against Q, then against V (up to 3 passes), expanded into G
    (T1.py:706-729)
The operator is the fused SpMM: H z - sigma z + shift Q_h^T Q_h z is one kernel.
With precision="mixed" the GMRES correction runs on the FP32 store (the
correction only needs a few digits); Ritz pairs, residuals, orthogonalisation
and G stay FP64.  Deviation: the Gram-Schmidt against locked vectors is done as
two classical passes (two matrix-vector products) instead of a vector-by-vector
modified loop; both leave z orthogonal to Q to working precision.
"""
from __future__ import annotations

import numpy as np
import torch

from ..krylov import HessianOperator


class _ShiftedOp:
    """x -> (H - sigma I) x + s Q^T Q x, FP64 interface."""

    def __init__(self, A, prec, Qh, shift):
        self.op = HessianOperator(A, prec=prec, Q=Qh, hot_shift=shift)
        self.n_spmm = 0

    def __call__(self, x, sigma, out=None):
        self.n_spmm += 1
        return self.op(x, out=out, gamma=-sigma)


def _gmres_deflate(matvec, b, x0, uu, tol, restart=20, maxiter=20):
    """Projected GMRES(restart) of IterativeSolvers.py:216-305 on the GPU; the
    small least-squares problem goes to the host as in the reference."""
    n = b.shape[0]
    dev = b.device
    x = x0.clone()
    b_norm = float(torch.linalg.vector_norm(b))
    if b_norm == 0:
        return b
    atol = tol * b_norm
    restart = min(restart, n)
    V = torch.empty((restart, n), dtype=torch.float64, device=dev)
    H = torch.zeros((restart + 1, restart), dtype=torch.float64, device=dev)
    e = np.zeros(restart + 1)
    iters = 0
    while True:
        mx = x - torch.dot(uu, x) * uu
        ax = matvec(mx)
        ax -= torch.dot(uu, ax) * uu
        r = b - ax
        r_norm = float(torch.linalg.vector_norm(r))
        if r_norm <= atol or iters >= maxiter:
            break
        v = r / r_norm
        V[0] = v
        e[0] = r_norm
        for j in range(restart):
            z = v - torch.dot(uu, v) * uu
            u = matvec(z)
            u -= torch.dot(uu, z) * uu
            Vj = V[:j + 1]
            h = Vj.mv(u)
            u -= Vj.t().mv(h)
            H[:j + 1, j] = h
            H[j + 1, j] = torch.linalg.vector_norm(u)
            if j + 1 < restart:
                v = u / H[j + 1, j]
                V[j + 1] = v
        y = np.linalg.lstsq(H.cpu().numpy(), e, rcond=None)[0]
        x += V.t().mv(torch.from_numpy(y).to(dev))
        iters += restart
    return mx


def jdm(A, k=16, tol=1e-10, maxiter=1000, correction_maxiter=20, workspace_factor=2, intermediate_tol=1e-3,
        gap=0.1, factoring_tol=1e-4, Q=None, shift=10.0, polynomial=None, precision="f64", seed=0,
        return_info=False, verbose=False):
    assert polynomial is None, ("ABORTED. WARNING. The J in JDM is targeting the smallest eigval due to implicit "
                                "inversion which counteract the goal of Cheb to map to the largest eigval. You are "
                                "advised to Use CDSI instead.")
    assert workspace_factor > 1, "ABORTED. User_WorkspaceSizeFactor: int > 1"
    assert precision in ("f64", "mixed"), "ABORTED. precision must be 'f64' or 'mixed'"
    N = A.shape[0]
    dev = A.device
    f64 = torch.float64
    jmax = k * workspace_factor
    jmin = min(N, k)
    Hop = HessianOperator(A, prec=64, Q=Q, hot_shift=shift)
    corr = _ShiftedOp(A, 32 if precision == "mixed" else 64, Hop.Q, shift)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    V = torch.zeros((jmax + 1, N), dtype=f64, device=dev)
    Qc = torch.zeros((jmin, N), dtype=f64, device=dev)
    eig = np.zeros(k)
    v0 = torch.rand(N, generator=g, dtype=f64, device=dev) - 0.5
    v0 /= torch.linalg.vector_norm(v0)
    Av = Hop(v0)
    V[0] = v0
    G = np.array([[float(torch.dot(v0, Av))]])
    nconv = 0
    jacc = 0
    jcur = 1
    n_outer_spmm = 1
    theta = G[0, 0]
    cur = np.inf
    for it in range(maxiter):
        S, W = np.linalg.eigh(G, UPLO="L")
        while True:
            theta = float(S[0])
            Wd = torch.from_numpy(np.ascontiguousarray(W)).to(dev)
            u = Wd[:, 0] @ V[:W.shape[0]]
            r = Hop(u)
            n_outer_spmm += 1
            r -= theta * u
            cur = float(torch.linalg.vector_norm(r))
            if verbose and it % 100 == 0:
                print(it, cur, theta, nconv)
            sigma = theta - gap
            Qc[jacc] = u
            jcur = W.shape[0]
            if cur > tol or (nconv != k - 1 and len(S) <= 1):
                break
            eig[nconv] = theta
            nconv += 1
            jacc += 1
            V[:W.shape[1] - 1] = Wd[:, 1:].t() @ V[:W.shape[0]]
            jcur = W.shape[1] - 1
            S = S[1:]
            G, W = np.diag(S), np.identity(S.shape[0])
            if nconv == k:
                idx = np.argsort(eig)
                out = (torch.from_numpy(eig[idx].copy()).to(dev), Qc[torch.from_numpy(idx).to(dev)].t().contiguous())
                if return_info:
                    return (*out, dict(iterations=it + 1, converged=True, n_spmm=corr.n_spmm + n_outer_spmm))
                return out
        if S.shape[0] == jmax:
            Wd = torch.from_numpy(np.ascontiguousarray(W[:, :jmin])).to(dev)
            V[:jmin] = Wd.t() @ V[:W.shape[0]]
            jcur = jmin
            S = S[:jmin]
            G, W = np.diag(S), np.identity(S.shape[0])
        sh = theta if cur < intermediate_tol else sigma
        uu = u / torch.linalg.vector_norm(u)
        ctol = cur * factoring_tol
        x0 = torch.rand(N, generator=g, dtype=f64, device=dev) * (ctol / N)
        z = _gmres_deflate(lambda x: corr(x, sh), -r, x0, uu, ctol, 20, correction_maxiter)
        Ql = Qc[:jacc + 1]
        for _ in range(2):
            z = z - Ql.t().mv(Ql.mv(z))
        Vc = V[:jcur]
        r_pre = float(torch.sqrt(torch.abs(torch.dot(z, z))))
        r1 = r_pre
        for _ in range(3):
            z = z - Vc.t().mv(Vc.mv(z))
            r1 = float(torch.sqrt(torch.abs(torch.dot(z, z))))
            if r1 > r_pre / 2:
                break
            r_pre = r1
        z = z / r1
        Az = Hop(z)
        n_outer_spmm += 1
        vaz = Vc.mv(Az).cpu().numpy()
        zaz = float(torch.dot(Az, z))
        G = np.block([[G, vaz[:, None]], [vaz[None, :], np.array([[zaz]])]])
        V[jcur] = z
    eig[nconv] = theta
    nconv += 1
    idx = np.argsort(eig)
    print("ABORTED. It did not actually converged! We went through %s coarse iter and collected %s converged"
          % (maxiter, nconv))
    out = (torch.from_numpy(eig[idx].copy()).to(dev), Qc[torch.from_numpy(idx).to(dev)].t().contiguous())
    if return_info:
        return (*out, dict(iterations=maxiter, converged=False, n_spmm=corr.n_spmm + n_outer_spmm))
    return out
