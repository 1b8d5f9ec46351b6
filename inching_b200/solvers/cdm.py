"""Chebyshev-Davidson eigensolver on the GPU.

Follows InchingLiteInteger/Burn/ChebyshevDavidsonSubspaceIteration/T1.py:229-623
(Zhou & Saad, "A Chebyshev-Davidson algorithm for large symmetric
eigenproblems", SIAM J. Matrix Anal. Appl. 29 (2007)):
  * the expansion vector is the current Ritz vector passed through the unscaled
    Chebyshev filter T_{m+1}((c - H)/e) on [low, high], low = the median active
    Ritz value of the previous step (at least the spectrum's lower bound), high =
    the spectrum's upper bound + 1e-5                       (T1.py:195-226, 384-396, 615)
  * it is orthogonalised against the basis V and appended; V, H V and the
    projected matrix G cover only the active (unconverged) columns
    (T1.py:400-451)
  * G's eigenproblem on the host (LAPACK); restart to
    max(nc + 1, k + 5, min(k + nc, jmax - 5)) columns when V is full
    (T1.py:455-486)
  * the first active Ritz pair is converged when ||H x - theta x|| < tol * beta,
    beta = the largest |theta| seen so far                   (T1.py:364-366, 495-533)

Every filter degree is one fused SpMM, X_{t+1} = a H X_t + g X_t + b X_{t-1};
the whole filter (m + 1 launches) is captured once as a CUDA graph whose
coefficients come from a device table, so each outer step replays one graph.

Differences from the reference, all of which keep its results:
  * after a convergence the next filter input is the next active Ritz vector
    (Zhou & Saad, Alg. 3.1); the reference filters the just-converged vector,
    whose filtered image Gram-Schmidt then reduces to rounding noise
    (T1.py:596-597);
  * several leading Ritz pairs may converge in one step (the reference tests one);
  * Gram-Schmidt is two classical passes against the whole basis (GEMVs), in
    place of one classical pass plus a modified pass over converged columns;
  * block=b > 1 filters the next b active Ritz vectors together (one SpMM of
    width b per degree; Zhou, J. Comput. Phys. 229 (2010), block variant);
  * Q (rows spanning modes to skip, e.g. the rigid-body basis) is projected out
    of every new vector; the reference refuses Hotelling deflation here
    (T1.py:257) and its facade keeps that refusal;
  * the restart size is clamped to the workspace (the reference's
    k + 5 exceeds jmax = 2k for k < 5);
  * precision="mixed" runs the filter on the FP32 store while the leading active
    residual is above MIXED_SWITCH * beta, then on the FP64 store: the expansion
    carries the Ritz vector's error, which FP32 rounding of the filtered vector
    buries once it falls below ~1e-7.  H V, G, Ritz pairs and residuals stay FP64,
    so the tolerance means the same in both precisions.
"""
from __future__ import annotations

import time

import numpy as np
import torch

from ..krylov import HessianOperator
from .chfsi import _GraphFilter


def filter_rows(degree, low, high):
    """Coefficient rows (a, g, b) of T_{degree+1}((c - H)/e) as a three-term
    recurrence: X_1 = (c X_0 - H X_0)/e, X_{t+1} = 2 (c X_t - H X_t)/e - X_{t-1}."""
    e = (high - low) / 2.0
    c = (high + low) / 2.0
    return [[-1.0 / e, c / e, 0.0]] + [[-2.0 / e, 2.0 * c / e, -1.0]] * degree


class _EagerRows:
    """The same recurrence launch by launch (stores without the segmented epilogue)."""

    def __init__(self, A, prec):
        self.A = A
        self.prec = prec
        self.n_spmm = 0
        self.replays = 0

    def run_rows(self, X64, rows):
        dt = torch.float64 if self.prec == 64 else torch.float32
        b = X64.shape[1]
        bp = (b + 7) // 8 * 8
        X = torch.zeros((X64.shape[0], bp), dtype=dt, device=X64.device)
        X[:, :b] = X64
        Y = torch.empty_like(X)
        a0, g0, _ = rows[0]
        self.A.matmul(X, out=Y, prec=self.prec, alpha=a0, gamma=g0)
        for a, g, bb in rows[1:]:
            self.A.matmul(Y, out=X, prec=self.prec, alpha=a, gamma=g, beta=bb, Yin=X)
            X, Y = Y, X
        self.n_spmm += len(rows)
        return Y[:, :b].to(torch.float64)


NOISE = 1e-13         # remainder (relative to the unit input) below which a column is rounding noise
MIXED_SWITCH = 1e-5   # leading residual / beta below which the mixed solver filters in FP64


def _orthonormalise(Z, V, Qd, gen):
    """Columns of Z (n, b) orthonormal to the rows of V (j, n) and Qd, and to each
    other.  The remainder after projection is legitimately small (about the size of
    the Ritz vector's error, which is what Davidson expands with); only a column
    reduced to rounding noise is replaced by a random one."""
    for attempt in range(4):
        if Qd is not None:
            for _ in range(2):
                Z = Z - Qd.t() @ (Qd @ Z)
        Z = Z / torch.linalg.vector_norm(Z, dim=0, keepdim=True).clamp_min(1e-300)
        for _ in range(2):
            Z = Z - V.t() @ (V @ Z)
            if Qd is not None:
                Z = Z - Qd.t() @ (Qd @ Z)
        bad = torch.linalg.vector_norm(Z, dim=0) < NOISE
        if not bool(bad.any()):
            Z = Z / torch.linalg.vector_norm(Z, dim=0, keepdim=True)
            Qz, R = torch.linalg.qr(Z)
            bad = torch.diagonal(R).abs() < NOISE
            if not bool(bad.any()):
                for _ in range(2):
                    Qz = Qz - V.t() @ (V @ Qz)
                return Qz / torch.linalg.vector_norm(Qz, dim=0, keepdim=True)
        Z = Z.clone()
        Z[:, bad] = torch.rand((Z.shape[0], int(bad.sum())), generator=gen, dtype=Z.dtype, device=Z.device) - 0.5
    raise RuntimeError("cdm: could not extend the basis (the space is exhausted)")


def cdm(A, k=16, tol=1e-10, maxiter=100000, workspace_factor=2, degree=80, spectrum_bound=None, Q=None,
        precision="f64", block=1, seed=0, cuda_graph=True, return_info=False, verbose=False):
    """k lowest eigenpairs of the store A (+PlusI), orthogonal to the rows of Q.

    spectrum_bound: (lower, upper) bound of the spectrum (e.g. from
    spectrum.estimate_spectrum_bound).  Returns eigenvalues (k,) ascending and
    eigenvectors (n, k), FP64 CUDA tensors."""
    t_start = time.perf_counter()
    assert spectrum_bound is not None, "ABORTED. The spectrum bound has to be initiated."
    assert workspace_factor > 1, "ABORTED. We require User_WorkspaceSizeFactor > 1 "
    assert precision in ("f64", "mixed"), "ABORTED. precision must be 'f64' or 'mixed'"
    assert block >= 1, "ABORTED. block must be >= 1"
    n = A.shape[0]
    dev = A.device
    f64 = torch.float64
    Qd = None if Q is None else HessianOperator(A, Q=Q).Q
    r = 0 if Qd is None else Qd.shape[0]
    jmin = min(n - r, k)
    assert jmin > 0, "ABORTED. k must be positive"
    bs = int(block)
    jmax = min(max(workspace_factor * jmin, jmin + bs + 5), n - r)
    op64 = HessianOperator(A, prec=64)
    graph_ok = cuda_graph and hasattr(A, "matmul_seg")
    filters = {}

    def filt_for(prec):
        if prec not in filters:
            filters[prec] = _GraphFilter(A, prec) if graph_ok else _EagerRows(A, prec)
        return filters[prec]
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)

    V = torch.zeros((jmax, n), dtype=f64, device=dev)     # basis rows
    AV = torch.zeros((jmax, n), dtype=f64, device=dev)    # H V rows
    G = np.zeros((jmax, jmax))
    thb = float(spectrum_bound[-1]) + 1e-5
    lower = float(spectrum_bound[0])

    Z = torch.rand((n, bs), generator=gen, dtype=f64, device=dev)
    Z = _orthonormalise(Z, V[:0], Qd, gen)
    V[:bs] = Z.t()
    AV[:bs] = op64(Z.contiguous()).t()
    G[:bs, :bs] = (V[:bs] @ AV[:bs].t()).cpu().numpy()
    G[:bs, :bs] = 0.5 * (G[:bs, :bs] + G[:bs, :bs].T)
    S, W = np.linalg.eigh(G[:bs, :bs])
    Wd = torch.from_numpy(W).to(dev)
    V[:bs] = Wd.t() @ V[:bs]
    AV[:bs] = Wd.t() @ AV[:bs]
    G[:bs, :bs] = np.diag(S)
    squeeze = (thb + S[0]) / 2.0
    beta = max(1e-14, float(np.max(np.abs(S))))
    nc = 0            # converged (locked) columns: V[:nc]
    j = bs            # basis size
    conv = []
    n_spmm_hv = bs
    it = 0
    converged = False
    lead_res = np.inf
    f32_steps = 0
    for it in range(maxiter):
        # ---- expansion: filter the next active Ritz vectors -------------------
        nb = min(bs, jmax - j)
        if j > nc:
            nb = min(nb, j - nc)
            X = V[nc:nc + nb].t().contiguous()
        else:       # every basis column converged: expand from random vectors
            X = torch.rand((n, nb), generator=gen, dtype=f64, device=dev) - 0.5
        prec = 32 if (precision == "mixed" and lead_res > MIXED_SWITCH * beta) else 64
        f32_steps += prec == 32
        Z = filt_for(prec).run_rows(X, filter_rows(degree, squeeze, thb))
        Z = _orthonormalise(Z, V[:j], Qd, gen)
        V[j:j + nb] = Z.t()
        AV[j:j + nb] = op64(Z.contiguous()).t()
        n_spmm_hv += nb
        jn = j + nb
        Gc = (V[nc:jn] @ AV[j:jn].t()).cpu().numpy()       # (jn - nc, nb)
        G[nc:jn, j:jn] = Gc
        G[j:jn, nc:jn] = Gc.T
        Ga = 0.5 * (G[nc:jn, nc:jn] + G[nc:jn, nc:jn].T)
        S, W = np.linalg.eigh(Ga)
        # ---- restart when the workspace cannot take another expansion ----------
        if jn + bs > jmax:
            jr = max(nc + 1, jmin + 5, min(jmin + nc, jmax - 5))
            jr = min(jr, jmax - bs, jn)
            jr = max(jr, nc + 1)
        else:
            jr = jn
        nn = jr - nc
        Wd = torch.from_numpy(np.ascontiguousarray(W[:, :nn])).to(dev)
        V[nc:jr] = Wd.t() @ V[nc:jn]
        AV[nc:jr] = Wd.t() @ AV[nc:jn]
        G[nc:jr, nc:jr] = np.diag(S[:nn])
        beta = max(beta, float(np.max(np.abs(S))))
        tolr = tol * beta
        # ---- convergence of the leading active Ritz pairs ----------------------
        cand = min(nn, jmin - nc, bs + 4)
        Rv = AV[nc:nc + cand] - torch.from_numpy(S[:cand].copy()).to(dev)[:, None] * V[nc:nc + cand]
        res = torch.linalg.vector_norm(Rv, dim=1).cpu().numpy()
        nl = 0
        while nl < cand and res[nl] < tolr:
            nl += 1
        lead_res = float(res[nl]) if nl < cand else np.inf
        if verbose and (it % 50 == 0 or nl):
            print(f"cdm it {it}: res {res[0]:.3e} theta {S[0]:.6f} converged {nc + nl}/{jmin} basis {jr}")
        conv.extend(S[:nl].tolist())
        nc += nl
        j = jr
        if nc >= jmin:
            converged = True
            break
        squeeze = max(float(np.median(S)), lower)
    if not converged:
        print(f"ABORTED. It did not actually converged! We went through {it + 1} coarse iter "
              f"and collected {nc} converged")
    lam = np.asarray(conv[:jmin])
    idx = np.argsort(lam)
    idx_t = torch.from_numpy(idx).to(dev)
    evals = torch.from_numpy(np.ascontiguousarray(lam[idx])).to(dev)
    evecs = V[:len(lam)][idx_t].t().contiguous()
    if return_info:
        if len(lam):
            Rf = op64(evecs) - evecs * evals[None, :]
            max_res = float(torch.linalg.vector_norm(Rf, dim=0).max()) / beta
        else:
            max_res = None
        info = dict(iterations=it + 1, converged=converged, n_spmm_hv=n_spmm_hv,
                    n_spmm_filter=sum(f.n_spmm for f in filters.values()),
                    filter_graph_replays=sum(f.replays for f in filters.values()), filter_f32_steps=f32_steps,
                    beta=beta, max_rel_residual=max_res, basis=jmax, block=bs, degree=degree,
                    seconds=time.perf_counter() - t_start)
        return evals, evecs, info
    return evals, evecs
