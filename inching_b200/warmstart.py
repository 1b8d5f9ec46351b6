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
                      return_info=False):
    """(3N, n_vectors) FP64 initial block whose columns are the lowest non-rigid
    bead modes prolonged to the atoms (atom order of X_nm)."""
    from .solvers.chfsi import chfsi
    pos, bead = bead_model(X_nm, bead_edge_A)
    nb = pos.shape[0]
    m = min(n_vectors, 3 * nb - 7)
    Hc = HessianStore(pos, rc_bead_A, plus_i=1.0)
    Qc = rigid_body_basis(pos)
    ev, Vc, info = chfsi(Hc, m, tol=tol, Q=Qc, precision="mixed", seed=seed + 7, return_info=True)
    Vb = Vc.reshape(nb, 3, m)
    del Vc, Hc
    V = Vb.index_select(0, bead).reshape(3 * X_nm.shape[0], m)
    if m < n_vectors:      # pad with random columns so the block has the requested width
        V = torch.cat([V, torch.randn((V.shape[0], n_vectors - m), dtype=V.dtype, device=V.device)], dim=1)
    if return_info:
        return V, dict(beads=int(nb), coarse_modes=m, coarse_iterations=info["iterations"],
                       coarse_seconds=info["seconds"])
    return V
