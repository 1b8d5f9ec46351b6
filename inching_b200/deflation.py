"""Rigid-body deflation basis for explicit (Hotelling) deflation.

Follows the drivers (Command8A/commandBenchmark_InchingTRLMHD_Linux_Pdb_0064_A100.py:
314-372): three unit translations, the three rotation fields X @ R_{x,y,z}
normalised, then two rounds of Gram-Schmidt (each vector projected twice).
These six vectors span the exact null space of the ANM Hessian, i.e. they are
eigenvectors of H + PlusI*I with eigenvalue PlusI."""
from __future__ import annotations

import numpy as np
import torch


def translation_basis(n_atoms: int, device="cuda") -> torch.Tensor:
    """(3, 3N) unit translations: the null space of an ANM with periodic xy
    images, where rotations are no longer zero modes (the many-mode notebook keeps
    only the three translations under PBC)."""
    Q = torch.zeros((3, n_atoms, 3), dtype=torch.float64, device=device)
    for a in range(3):
        Q[a, :, a] = 1.0 / np.sqrt(n_atoms)
    return Q.reshape(3, 3 * n_atoms)


def rigid_body_basis(X_nm, device=None) -> torch.Tensor:
    """(6, 3N) float64 orthonormal rows on the device of X (or `device`)."""
    if isinstance(X_nm, torch.Tensor):
        X = X_nm.to(dtype=torch.float64, device=device or X_nm.device)
    else:
        X = torch.from_numpy(np.asarray(X_nm, dtype=np.float64)).to(device or "cuda")
    n = X.shape[0]
    Q = torch.zeros((6, 3 * n), dtype=torch.float64, device=X.device)
    for i in range(3):
        q = torch.zeros((n, 3), dtype=torch.float64, device=X.device)
        q[:, i] = 1.0 / np.sqrt(n)
        Q[i] = q.reshape(-1)
    R = [torch.tensor(m, dtype=torch.float64, device=X.device).t() for m in (
        [[0, 0, 0], [0, 0, -1], [0, 1, 0]], [[0, 0, 1], [0, 0, 0], [-1, 0, 0]], [[0, -1, 0], [1, 0, 0], [0, 0, 0]])]
    for t in range(3):
        g = (X @ R[t]).reshape(-1)
        Q[3 + t] = g / torch.linalg.vector_norm(g)
    V = Q.t().contiguous()
    for _ in range(2):
        for ix in range(1, 6):
            for _twice in range(2):
                V[:, ix] -= V[:, :ix] @ (V[:, :ix].t() @ V[:, ix])
                V[:, ix] /= torch.sqrt(V[:, ix] @ V[:, ix])
    return V.t().contiguous()


def rigid_body_basis_padded(X_nm: torch.Tensor, atom_offsets, n_max_dof: int) -> torch.Tensor:
    """Rigid-body bases of many structures at once: X_nm holds the structures'
    atoms back to back (atom_offsets, S+1); returns (S, 6, n_max_dof) with each
    structure's six orthonormal rows (same construction as rigid_body_basis,
    batched over structures; padding is zero)."""
    dev = X_nm.device
    off = torch.as_tensor(np.asarray(atom_offsets), device=dev)
    S = off.numel() - 1
    sizes = (off[1:] - off[:-1])
    n_atoms_max = n_max_dof // 3
    sid = torch.repeat_interleave(torch.arange(S, device=dev), sizes)
    local = torch.arange(X_nm.shape[0], device=dev) - off[:-1][sid]
    Xp = torch.zeros((S, n_atoms_max, 3), dtype=torch.float64, device=dev)
    Xp[sid, local] = X_nm
    mask = torch.zeros((S, n_atoms_max, 1), dtype=torch.float64, device=dev)
    mask[sid, local] = 1.0
    V = torch.zeros((S, 6, n_atoms_max, 3), dtype=torch.float64, device=dev)
    inv = (1.0 / torch.sqrt(sizes.double()))[:, None]
    for i in range(3):
        V[:, i, :, i] = inv * mask[:, :, 0]
    R = [torch.tensor(m, dtype=torch.float64, device=dev).t() for m in (
        [[0, 0, 0], [0, 0, -1], [0, 1, 0]], [[0, 0, 1], [0, 0, 0], [-1, 0, 0]], [[0, -1, 0], [1, 0, 0], [0, 0, 0]])]
    for t in range(3):
        g = (Xp @ R[t]) * mask
        V[:, 3 + t] = g / torch.linalg.vector_norm(g.reshape(S, -1), dim=1)[:, None, None]
    V = V.reshape(S, 6, -1)
    for _ in range(2):
        for ix in range(1, 6):
            for _twice in range(2):
                c = torch.einsum("srn,sn->sr", V[:, :ix], V[:, ix])
                V[:, ix] -= torch.einsum("sr,srn->sn", c, V[:, :ix])
                V[:, ix] /= torch.linalg.vector_norm(V[:, ix], dim=1, keepdim=True)
    out = torch.zeros((S, 6, n_max_dof), dtype=torch.float64, device=dev)
    out[:, :, :V.shape[2]] = V
    return out
