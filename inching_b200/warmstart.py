"""Warm start for the block eigensolver from a coarse bead model (no reference
counterpart; the reference always starts from a random vector).

Atoms are pooled into beads by a cubic grid of edge `bead_edge_A` (about a
dozen atoms per bead at protein density); the beads form their own ANM with the
longer cutoff `rc_bead_A`, whose lowest modes are computed with the same GPU
block solver (loose tolerance, mixed precision).  Each bead mode is prolonged to
the atoms (every atom moves with its bead) and the block is handed to the fine
solver as its initial subspace, which then only has to correct the
intra-bead detail.  Everything runs on the GPU with the package's own kernels
(neighbour search, Hessian store, SpMM).
"""
from __future__ import annotations

import warnings

import torch

from .deflation import rigid_body_basis
from .hessian import HessianStore


def bead_model(X_nm: torch.Tensor, bead_edge_A=6.0):
    """(bead coordinates (nb, 3) nm, bead index of every atom (N,))."""
    edge = bead_edge_A / 10.0
    lo = X_nm.min(dim=0).values
    c = torch.floor((X_nm - lo) / edge).long()
    dims = c.max(dim=0).values + 1
    key = (c[:, 0] * dims[1] + c[:, 1]) * dims[2] + c[:, 2]
    uniq, bead = torch.unique(key, return_inverse=True)
    nb = uniq.shape[0]
    cnt = torch.zeros(nb, dtype=torch.float64, device=X_nm.device).index_add_(
        0, bead, torch.ones_like(bead, dtype=torch.float64))
    pos = torch.zeros((nb, 3), dtype=torch.float64, device=X_nm.device).index_add_(0, bead, X_nm)
    return pos / cnt[:, None], bead


def coarse_warm_start(X_nm: torch.Tensor, n_vectors: int, bead_edge_A=6.0, rc_bead_A=12.0, tol=1e-4, seed=0,
                      return_info=False, wanted=None):
    """(3N, n_vectors) FP64 initial block whose columns are the lowest non-rigid
    bead modes prolonged to the atoms (atom order of X_nm).

    wanted: how many of those bead modes the coarse solve converges (default all).
    The remaining columns are the coarse solver's own guard vectors, its
    unconverged Ritz vectors, which is all a fine solver's guard needs: for 256
    modes of 100k atoms (block 320) that makes the coarse block 320 columns wide
    instead of 400 and the warm start 37 ms instead of 53 ms, with the same 4 fine
    iterations.  For 1,000 modes of 2.4M atoms (block 1,250) converging all of them
    paid instead: 4 fine iterations and 93 s against 5 and 96 s.  No FP64
    certificate is taken on the coarse modes."""
    from .solvers.chfsi import chfsi
    pos, bead = bead_model(X_nm, bead_edge_A)
    nb = pos.shape[0]
    m = min(n_vectors, 3 * nb - 7)
    kc = m if wanted is None else max(1, min(int(wanted), m))
    Hc = HessianStore(pos, rc_bead_A, plus_i=1.0)
    Qc = rigid_body_basis(pos)
    ev, Vc, info = chfsi(Hc, kc, tol=tol, Q=Qc, precision="mixed", seed=seed + 7, guard=m - kc if kc < m else None,
                         final_f64=False, return_block=kc < m, return_info=True)
    Vb = Vc.reshape(nb, 3, m)
    del Vc, Hc
    V = Vb.index_select(0, bead).reshape(3 * X_nm.shape[0], m)
    if m < n_vectors:      # pad with random columns so the block has the requested width
        V = torch.cat([V, torch.randn((V.shape[0], n_vectors - m), dtype=V.dtype, device=V.device)], dim=1)
    if return_info:
        return V, dict(beads=int(nb), coarse_modes=m, coarse_converged=kc, coarse_iterations=info["iterations"],
                       coarse_seconds=info["seconds"])
    return V


# ---------------------------------------------------------------------------
# Galerkin bead start: the fine Hessian restricted to bead motions
# ---------------------------------------------------------------------------
class GalerkinOperator:
    """S = M^{-1/2} (P^T H P) M^{-1/2} for the piecewise-constant prolongation P
    (every atom moves with its bead) and M = P^T P (atoms per bead), as a cuSPARSE
    CSR matrix in FP64 and FP32, with the store's matmul interface (fused
    alpha / gamma / beta / accumulate epilogue) so the block solver runs on it.

    Built from the fine rank-one store: the (a, b) block of P^T H P is minus the
    sum of w w^T over atom pairs (i in a, j in b); the (a, a) block sums w w^T over
    the pairs leaving bead a, plus PlusI times the bead's atom count (pairs inside
    a bead cancel).  The eigenvectors of S, prolonged as P M^{-1/2} z, are the
    Rayleigh-Ritz vectors of H over the span of bead motions -- the best
    bead-motion block for H, which no bead spring model can beat."""

    def __init__(self, H, bead, nb, counts):
        dev = H.device
        n_at = H.n_atoms
        rows = torch.repeat_interleave(torch.arange(n_at, device=dev), torch.diff(H.rowptr))
        ent = H.ent64 if H.ent64 is not None else H.ent32.double()
        cols = H.cols.long()
        a, b = bead[rows], bead[cols]
        cross = a != b
        w = ent[cross, :3]
        a, b = a[cross], b[cross]
        del rows, cols, cross
        comps = torch.stack([w[:, 0] * w[:, 0], w[:, 1] * w[:, 1], w[:, 2] * w[:, 2],
                             w[:, 0] * w[:, 1], w[:, 0] * w[:, 2], w[:, 1] * w[:, 2]], dim=1)
        del w
        key = a * nb + b
        uk, inv = torch.unique(key, return_inverse=True)
        S = torch.zeros((uk.shape[0], 6), dtype=torch.float64, device=dev).index_add_(0, inv, comps)
        D = torch.zeros((nb, 6), dtype=torch.float64, device=dev).index_add_(0, a, comps)
        del comps, key, inv, a, b
        idx = torch.tensor([[0, 3, 4], [3, 1, 5], [4, 5, 2]], device=dev)
        ua, ub = uk // nb, uk % nb
        cnt = counts.to(torch.float64)
        off = -S[:, idx] / torch.sqrt(cnt[ua] * cnt[ub])[:, None, None]
        eye = torch.eye(3, dtype=torch.float64, device=dev)
        diag = (D[:, idx] + float(H.plus_i) * cnt[:, None, None] * eye) / cnt[:, None, None]
        brow = torch.cat([ua, torch.arange(nb, device=dev)])
        bcol = torch.cat([ub, torch.arange(nb, device=dev)])
        vals = torch.cat([off, diag]).reshape(-1)
        r3 = torch.arange(3, device=dev)
        R = (3 * brow[:, None, None] + r3[None, :, None]).expand(-1, 3, 3).reshape(-1)
        C = (3 * bcol[:, None, None] + r3[None, None, :]).expand(-1, 3, 3).reshape(-1)
        n = 3 * nb
        with warnings.catch_warnings():      # torch flags its sparse CSR support as beta
            warnings.simplefilter("ignore", UserWarning)
            coo = torch.sparse_coo_tensor(torch.stack([R, C]), vals, (n, n), check_invariants=False).coalesce()
            self.csr64 = coo.to_sparse_csr()
            self.csr32 = torch.sparse_csr_tensor(self.csr64.crow_indices(), self.csr64.col_indices(),
                                                 self.csr64.values().float(), (n, n))
        self.shape = (n, n)
        self.ndim = 2
        self.device = dev
        self.dtype = torch.float64
        self.plus_i = float(H.plus_i)
        self.n_atoms = nb

    def matmul(self, X, out=None, prec=None, alpha=1.0, gamma=0.0, beta=0.0, Yin=None, acc=None, mu=0.0, Q=None,
               hot_shift=0.0):
        if prec is None:
            prec = 64 if X.dtype == torch.float64 else 32
        S = self.csr64 if prec == 64 else self.csr32
        X2 = X if X.dim() == 2 else X[:, None]
        y = S @ X2
        if alpha != 1.0:
            y = alpha * y
        if gamma != 0.0:
            y = y + gamma * X2
        if Yin is not None and beta != 0.0:
            y = y + beta * (Yin if Yin.dim() == 2 else Yin[:, None])
        if Q is not None and hot_shift != 0.0:
            q = Q.to(X2.dtype)
            y = y + hot_shift * (q.t() @ (q @ X2))
        if X.dim() == 1:
            y = y[:, 0]
        if acc is not None:
            acc += mu * y
        if out is None:
            return y
        out.copy_(y)
        return out


def galerkin_warm_start(H, n_vectors, bead_edge_A=6.0, tol=1e-3, seed=0, return_info=False):
    """(3N, n_vectors) FP64 initial block: the lowest non-rigid eigenvectors of the
    Galerkin bead operator of the fine store H (atoms in H's order), prolonged to
    the atoms.  The six lowest coarse modes (the rigid-body motions, exact for
    translations) are dropped; the fine solver deflates the rigid basis itself."""
    from .solvers.chfsi import chfsi
    import time as _t
    t0 = _t.perf_counter()
    pos, bead = bead_model(H.X, bead_edge_A)
    nb = pos.shape[0]
    counts = torch.bincount(bead, minlength=nb)
    G = GalerkinOperator(H, bead, nb, counts)
    m = min(n_vectors + 6, 3 * nb - 1)
    _, Z, info = chfsi(G, m, tol=tol, precision="mixed", seed=seed + 11, return_info=True)
    Z = Z[:, 6:] if m > 6 else Z
    scale = 1.0 / torch.sqrt(counts.to(torch.float64))
    V = (Z.reshape(nb, 3, -1) * scale[:, None, None]).index_select(0, bead).reshape(3 * H.n_atoms, -1)
    if V.shape[1] < n_vectors:
        V = torch.cat([V, torch.randn((V.shape[0], n_vectors - V.shape[1]), dtype=V.dtype, device=V.device)], dim=1)
    if return_info:
        return V, dict(beads=int(nb), coarse_modes=int(Z.shape[1]), coarse_iterations=info["iterations"],
                       coarse_nnz=int(G.csr64.values().numel()), seconds=_t.perf_counter() - t0)
    return V
