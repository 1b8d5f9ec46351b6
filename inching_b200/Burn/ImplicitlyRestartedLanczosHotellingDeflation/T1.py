"""Drop-in for InchingLiteInteger.Burn.ImplicitlyRestartedLanczosHotellingDeflation.T1
(IRLM, T1.py:308-477).  Same signature as the reference; its one-argument operator
construction (T1.py:368) is replaced by the store's own operator.  Returns torch
CUDA tensors: eigenvalues (k,) ascending incl. PlusI and eigenvectors (n, k)."""
from __future__ import annotations

from ...solvers.irlm import irlm


def S_HeigvalIRLMHD_HeigvecIRLMHD(A, k=32, maxiter=15000, tol=1e-8, User_HalfMemMode=True,
                                  User_Q_HotellingDeflation=None, User_HotellingShift=10.0, User_Precision="f64",
                                  User_Seed=0):
    return irlm(A, k=k, maxiter=maxiter, tol=tol, Q=User_Q_HotellingDeflation, shift=User_HotellingShift,
                precision=User_Precision, seed=User_Seed)
