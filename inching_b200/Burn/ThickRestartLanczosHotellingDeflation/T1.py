"""Drop-in for InchingLiteInteger.Burn.ThickRestartLanczosHotellingDeflation.T1
(TRLM, T1.py:60-310).  Returns torch CUDA tensors in the reference's layout:
eigenvalues (k,) ascending including PlusI, eigenvectors (n, k) as columns."""
from __future__ import annotations

from ...solvers.trlm import trlm


def S_HeigvalTRLMHD_HeigvecTRLMHD(A, A_diag, k=32, maxiter=10000, tol=0, User_HalfMemMode=True,
                                  User_WorkspaceSizeFactor=2, User_Q_HotellingDeflation=None,
                                  User_HotellingShift=10.0, User_PolynomialParams=None, User_Precision="f64",
                                  User_Seed=0):
    """User_Precision: "f64" (reference arithmetic) or "mixed" (FP32 store and
    products, FP64 Lanczos basis, reorthogonalisation and Ritz values)."""
    return trlm(A, k=k, maxiter=maxiter, tol=tol, workspace_factor=User_WorkspaceSizeFactor,
                Q=User_Q_HotellingDeflation, shift=User_HotellingShift, polynomial=User_PolynomialParams,
                precision=User_Precision, seed=User_Seed)
