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
from .chfsi import _Phases


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


class _FilterSeg:
    """Scaled Chebyshev filter with each structure's own interval [a_s, b] and
    normalisation point a0_s; every degree is one segmented SpMM launch (per
    64-column panel) for all structures of the block-diagonal store."""

    def __init__(self, A, prec, atom_seg):
        self.A = A
        self.prec = prec
        self.atom_seg = atom_seg
        self.n_spmm = 0

    def __call__(self, X64, m, a, b, a0):
        a = np.asarray(a, dtype=np.float64)
        a0 = np.asarray(a0, dtype=np.float64)
        e = (b - a) / 2.0
        c = (b + a) / 2.0
        sigma = e / (a0 - c)
        sigma1 = sigma.copy()
        tau = 2.0 / sigma1
        coefs = [np.stack([sigma1 / e, -sigma1 * c / e, np.zeros_like(e)], axis=1)]
        for _ in range(2, m + 1):
            s2 = 1.0 / (tau - sigma)
            coefs.append(np.stack([2.0 * s2 / e, -2.0 * s2 * c / e, -sigma * s2], axis=1))
            sigma = s2
        table = torch.from_numpy(np.ascontiguousarray(np.stack(coefs))).to(X64.device)      # (m, S, 3)
        dt = torch.float64 if self.prec == 64 else torch.float32
        nb = X64.shape[1]
        bp = (nb + 7) // 8 * 8
        X = torch.zeros((X64.shape[0], bp), dtype=dt, device=X64.device)
        X[:, :nb] = X64
        Y = torch.empty_like(X)
        self.A.matmul_seg(X, Y, self.atom_seg, table[0], prec=self.prec)
        self.n_spmm += 1
        for t in range(1, m):
            self.A.matmul_seg(Y, X, self.atom_seg, table[t], Yin=X, prec=self.prec)
            X, Y = Y, X
            self.n_spmm += 1
        return Y[:, :nb].to(torch.float64)


def _eigh_small(G):
    """Batched symmetric eigensolve of the small (S, p, p) projected matrices: the
    package's one-CTA-per-matrix Jacobi kernel for p <= 64 (a few hundred us for a
    bucket), host LAPACK above that (cuSOLVER's batched solver took ~45 ms per call
    here, host numpy ~0.3 ms per 64 x 64 matrix)."""
    if G.is_cuda and G.shape[-1] <= 64:
        from .. import _native
        return _native.eigh_batched_small(G.contiguous())
    w, V = np.linalg.eigh(G.cpu().numpy())
    return torch.from_numpy(w).to(G.device), torch.from_numpy(V).to(G.device)


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


def batched_guard(k):
    """Guard vectors of the batched solve: at least max(16, k/2), then up to a
    multiple of 32 columns.  The SpMM runs 32/64-column panels, so a block that
    fills them costs little more per step and converges in fewer (512 structures,
    k = 32: 64 columns, 3.0 s and at most 5 iterations per bucket, against 48
    columns, 3.95 s and up to 8)."""
    p0 = k + max(16, int(math.ceil(0.5 * k)))
    return (p0 + 31) // 32 * 32 - k


def chfsi_batched(H, dof_offsets, k, tol=1e-6, Qp=None, precision="mixed", degree=24, guard=None, maxiter=200,
                  seed=0, verbose=False, profile=False, Y0=None):
    """Lowest k modes (orthogonal to Qp) of every diagonal block of H.

    dof_offsets: (S+1,) dof offsets of the structures inside H (block-diagonal).
    Qp: (S, r, n_max) padded deflation rows per structure or None.
    Returns (evals (S, k) FP64, vecs (n_total, k) FP64 with each structure's
    rows, info)."""
    dev = H.device
    ph = _Phases(profile)
    with ph("segments"):
        seg = _Segments(dof_offsets, dev)
    S = seg.S
    prec = 32 if precision == "mixed" else 64
    if guard is None:
        guard = batched_guard(k)
    p = min(k + guard, int(seg.sizes.min()) - (0 if Qp is None else Qp.shape[1]))
    assert p > k, "ABORTED. a structure is too small for k modes plus guard vectors"
    with ph("bound"):
        lo, hi = estimate_spectrum_bound(H, steps=40, seed=seed + 1, precision=precision)
    b_up = hi * 1.02 + 1e-3 * abs(hi)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    Y = torch.randn((seg.n_total, p), generator=g, dtype=torch.float64, device=dev)
    if Y0 is not None:
        c0 = min(Y0.shape[1], p)
        Y[:, :c0] = Y0[:, :c0]
    P = seg.gather(Y)
    if Qp is not None:
        P = _project_b(P, Qp)
    P = _cholqr_b(P) * seg.mask
    atom_sizes = torch.from_numpy(seg.sizes // 3).to(dev)
    atom_seg = torch.repeat_interleave(torch.arange(S, dtype=torch.int32, device=dev), atom_sizes).contiguous()
    filt = _FilterSeg(H, prec, atom_seg)
    it = 0
    th = None
    res = None
    for it in range(maxiter):
        with ph("rr_spmm"):
            Y = seg.scatter(P)
            if prec == 64:
                HY = H.matmul(Y.contiguous(), prec=64)
            else:
                HY = H.matmul(Y.to(torch.float32).contiguous(), prec=32).to(torch.float64)
            HP = seg.gather(HY)
        with ph("rr_gemm"):
            G = P.transpose(1, 2) @ HP
            G = 0.5 * (G + G.transpose(1, 2))
        with ph("rr_eigh"):
            th, W = _eigh_small(G)
        with ph("rr_rotate"):
            P = P @ W
            HP = HP @ W
            R = HP - P * th[:, None, :]
            res = torch.linalg.vector_norm(R, dim=1)                      # (S, p)
            worst = float((res[:, :k] / b_up).max())
        if verbose:
            print(f"batched it {it}: worst rel residual {worst:.2e}")
        if worst <= tol:
            break
        # each structure filters with its own interval: [largest block Ritz value, b]
        a = th[:, -1].cpu().numpy()
        a0 = th[:, 0].cpu().numpy()
        bad = ~((a0 < a) & (a < b_up))
        a = np.minimum(a, 0.999 * b_up)
        a0 = np.where(bad, a - 1e-3 * np.abs(a), a0)
        with ph("filter"):
            Z = filt(seg.scatter(P), degree, a, b_up, a0 - 1e-12)
            P = seg.gather(Z)
        with ph("orth"):
            if Qp is not None:
                P = _project_b(P, Qp)
            P = _cholqr_b(P) * seg.mask
    # final FP64 Rayleigh-Ritz of each structure's block; keep the k lowest
    Y = seg.scatter(P)
    HP = seg.gather(H.matmul(Y.contiguous(), prec=64))
    G = P.transpose(1, 2) @ HP
    G = 0.5 * (G + G.transpose(1, 2))
    th, W = _eigh_small(G)
    thk = th[:, :k].contiguous()
    Pk = P @ W[:, :, :k]
    R = HP @ W[:, :, :k] - Pk * thk[:, None, :]
    rel = torch.linalg.vector_norm(R, dim=1) / b_up
    info = dict(iterations=it + 1, n_spmm_filter=filt.n_spmm, block=p, degree=degree, structures=S,
                max_rel_residual=float(rel.max()), normH=b_up, phases_ms=ph.summary())
    return thk, seg.scatter(Pk), info
