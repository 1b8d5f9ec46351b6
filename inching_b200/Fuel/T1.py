"""Drop-in for InchingLiteInteger.Fuel.T1.Xnumpy_SparseCupyMatrixUngappped
(Fuel/T1.py:60-660): ANM Hessian assembly.  ReturnCupyHLowerTriangleInt32/Int64
return (A, A_diag) where A is the GPU Hessian store (shape/dtype/ndim like the
reference's CSR matrix) and A_diag the (3N,) float64 diagonal of H + PlusI*I.

The reference's row batches, ungapped column slices and int32/int64 CSR index
variants only organise its dense-batch assembly; the store built here does not
need them, so batch_head / maxleafsize / NnzMinMaxDict are accepted and ignored
and both Return* methods give the same object (column indices are int32 per atom
block, i.e. valid up to 2^31 atoms)."""
from __future__ import annotations

import torch

from ..hessian import HessianStore


class Xnumpy_SparseCupyMatrixUngappped:
    def __init__(self, X, batch_head=None, maxleafsize=100, rc_Gamma=8.0, device=None, User_PlusI=1.0,
                 dtype_temp=torch.float64, X_precision=None, NnzMinMaxDict=None, User_DictCharmmGuiPbc=None,
                 User_StorePrecisions=("f64", "f32")):
        self.pbc = None
        if User_DictCharmmGuiPbc is not None:
            from ..graph import pbc_box
            self.pbc = pbc_box(User_DictCharmmGuiPbc)
            assert self.pbc[0] > rc_Gamma / 10.0, "ABORTED. The PBC box size X is smaller than rc gamma."
            assert self.pbc[1] > rc_Gamma / 10.0, "ABORTED. The PBC box size Y is smaller than rc gamma."
        if isinstance(device, int):
            device = torch.device("cuda", device)
        self.X = X
        self.rc_Gamma = rc_Gamma / 10.0
        self.n_atoms = int(X.shape[0])
        self.User_PlusI = User_PlusI
        self.device = device
        self.precisions = User_StorePrecisions
        self._store = None

    def _build(self):
        if self._store is None:
            self._store = HessianStore(self.X, self.rc_Gamma * 10.0, plus_i=self.User_PlusI,
                                       precisions=self.precisions, device=self.device, pbc=self.pbc)
        return self._store

    def ReturnNumberTotalBatch(self):
        return 1

    def ReturnCupyHLowerTriangleInt32(self, User_MaxHalfNnzBufferSize=1e8):
        A = self._build()
        return A, A.A_diag

    def ReturnCupyHLowerTriangleInt64(self, User_MaxHalfNnzBufferSize=1e8):
        A = self._build()
        return A, A.A_diag
