"""Rigid-body deflation basis for explicit (Hotelling) deflation.

Follows the drivers (Command8A/commandBenchmark_InchingTRLMHD_Linux_Pdb_0064_A100.py:
314-372): three unit translations, the three rotation fields X @ R_{x,y,z}
normalised, then two rounds of Gram-Schmidt (each vector projected twice).
These six vectors span the exact null space of the ANM Hessian, i.e. they are
eigenvectors of H + PlusI*I with eigenvalue PlusI."""
from __future__ import annotations

import numpy as np
import torch


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
