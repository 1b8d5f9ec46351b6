"""Drop-in for InchingLiteInteger.Burn.Orthogonalization.T3 (T3.py:62-164): the
Hotelling update res += shift * Q^T (Q x).  The solvers fuse this into the SpMM
epilogue; this standalone form serves callers of the reference function."""
from __future__ import annotations

import torch


def T3_QHotelling_x_Ax_HotelledAx(QHotelling, x, res, HotellingShift=10.0):
    Q = QHotelling
    if not isinstance(Q, torch.Tensor):
        import numpy as np
        import scipy.sparse as sp
        Q = torch.from_numpy(np.asarray(Q.toarray() if sp.issparse(Q) else Q, dtype=np.float64)).to(x.device)
    xv = x.reshape(-1)
    res.reshape(-1).add_(HotellingShift * (Q.t() @ (Q @ xv)))
    return res
