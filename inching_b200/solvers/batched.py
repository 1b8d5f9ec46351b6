"""Many structures in one solve: block-diagonal batched Chebyshev-filtered
subspace iteration (no reference counterpart; the reference loops over
structures one at a time, e.g. Command8A/commandBenchmark_InchingTRLMHD_Linux_Pdb_0064_A100.py:189).

The structures of one batch share ONE Hessian store: their coordinates are laid
out on a lattice far enough apart that no pair crosses structures, so H is
block-diagonal and one SpMM launch (per 64-column panel) applies every
structure's Hessian to its own block of the (n_total, p) multivector.  Each
Chebyshev degree is therefore one launch for the whole batch.  The per-structure
parts -- deflation of the six rigid-body vectors, Cholesky-QR, Rayleigh-Ritz and
residuals -- run as batched GEMMs / batched eigh on a padded (S, n_max, p) view.
Filter bounds are common to the batch (largest block Ritz value and spectrum
bound over its structures), which is why callers bucket structures of similar
size together (see inching_b200.batched).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from ..spectrum import estimate_spectrum_bound
from .chfsi import _Filter


class _Segments:
    """Padded view of a row-segmented (n_total, p) block: gather to (S, n_max, p)
    and scatter back, with padding rows reading a zero row."""

    def __init__(self, dof_offsets, device):
        off = np.asarray(dof_offsets, dtype=np.int64)
        self.S = len(off) - 1
        self.sizes = np.diff(off)
        self.n_max = int(self.sizes.max())
        n_total = int(off[-1])
        idx = np.full((self.S, self.n_max), n_total, dtype=np.int64)      # n_total -> zero row
        back = np.empty(n_total, dtype=np.int64)
        for s in range(self.S):
            n = self.sizes[s]
            idx[s, :n] = np.arange(off[s], off[s + 1])
            back[off[s]:off[s + 1]] = s * self.n_max + np.arange(n)
        self.idx = torch.from_numpy(idx.reshape(-1)).to(device)
        self.back = torch.from_numpy(back).to(device)
        self.n_total = n_total
        mask = np.zeros((self.S, self.n_max, 1))
        for s in range(self.S):
            mask[s, :self.sizes[s]] = 1.0
        self.mask = torch.from_numpy(mask).to(device)

    def gather(self, Y):
        Z = torch.cat([Y, torch.zeros((1, Y.shape[1]), dtype=Y.dtype, device=Y.device)], dim=0)
        return Z.index_select(0, self.idx).reshape(self.S, self.n_max, Y.shape[1])

    def scatter(self, P):
        return P.reshape(self.S * self.n_max, P.shape[2]).index_select(0, self.back)


def _cholqr_b(P):
    for _ in range(2):
        G = P.transpose(1, 2) @ P
        L = torch.linalg.cholesky(G, upper=True)
        P = torch.linalg.solve_triangular(L, P, upper=True, left=False)
    return P


def _project_b(P, Qp):
    """P (S, n, p) minus Qp^T (Qp P), Qp (S, r, n) orthonormal rows; twice."""
    for _ in range(2):
        P = P - Qp.transpose(1, 2) @ (Qp @ P)
    return P


def chfsi_batched(H, dof_offsets, k, tol=1e-6, Qp=None, precision="mixed", degree=24, guard=None, maxiter=200,
                  seed=0, verbose=False):
    """Lowest k modes (orthogonal to Qp) of every diagonal block of H.

    dof_offsets: (S+1,) dof offsets of the structures inside H (block-diagonal).
    Qp: (S, r, n_max) padded deflation rows per structure or None.
    Returns (evals (S, k) FP64, vecs (n_total, k) FP64 with each structure's
    rows, info)."""
    dev = H.device
    seg = _Segments(dof_offsets, dev)
    S = seg.S
    prec = 32 if precision == "mixed" else 64
    if guard is None:
        guard = max(12, int(math.ceil(0.3 * k)))
    p = min(k + guard, int(seg.sizes.min()) - (0 if Qp is None else Qp.shape[1]))
    assert p > k, "ABORTED. a structure is too small for k modes plus guard vectors"
    lo, hi = estimate_spectrum_bound(H, steps=40, seed=seed + 1, precision=precision)
    b_up = hi * 1.02 + 1e-3 * abs(hi)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    Y = torch.randn((seg.n_total, p), generator=g, dtype=torch.float64, device=dev)
    P = seg.gather(Y)
    if Qp is not None:
        P = _project_b(P, Qp)
    P = _cholqr_b(P) * seg.mask
    filt = _Filter(H, prec)
    it = 0
    th = None
    res = None
    for it in range(maxiter):
        Y = seg.scatter(P)
        if prec == 64:
            HY = H.matmul(Y.contiguous(), prec=64)
        else:
            HY = H.matmul(Y.to(torch.float32).contiguous(), prec=32).to(torch.float64)
        HP = seg.gather(HY)
        G = P.transpose(1, 2) @ HP
        G = 0.5 * (G + G.transpose(1, 2))
        th, W = torch.linalg.eigh(G)
        P = P @ W
        HP = HP @ W
        R = HP - P * th[:, None, :]
        res = torch.linalg.vector_norm(R, dim=1)                      # (S, p)
        worst = float((res[:, :k] / b_up).max())
        if verbose:
            print(f"batched it {it}: worst rel residual {worst:.2e}")
        if worst <= tol:
            break
        a = float(th[:, -1].max())
        a0 = float(th[:, 0].min())
        if not (a0 < a < b_up):
            a0 = a - 1e-3 * abs(a)
        Z = filt(seg.scatter(P), degree, a, b_up, a0 - 1e-12)
        P = seg.gather(Z)
        if Qp is not None:
            P = _project_b(P, Qp)
        P = _cholqr_b(P) * seg.mask
    # final FP64 Rayleigh-Ritz of each structure's block; keep the k lowest
    Y = seg.scatter(P)
    HP = seg.gather(H.matmul(Y.contiguous(), prec=64))
    G = P.transpose(1, 2) @ HP
    G = 0.5 * (G + G.transpose(1, 2))
    th, W = torch.linalg.eigh(G)
    thk = th[:, :k].contiguous()
    Pk = P @ W[:, :, :k]
    R = HP @ W[:, :, :k] - Pk * thk[:, None, :]
    rel = torch.linalg.vector_norm(R, dim=1) / b_up
    info = dict(iterations=it + 1, n_spmm_filter=filt.n_spmm, block=p, degree=degree, structures=S,
                max_rel_residual=float(rel.max()), normH=b_up)
    return thk, seg.scatter(Pk), info
