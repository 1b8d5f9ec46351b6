"""Drop-in for InchingLiteInteger.Burn.ChebyshevDavidsonSubspaceIteration.T1
(CDM, T1.py:229-623; spectrum bound helpers T1.py:81-192).  Returns torch CUDA
tensors: eigenvalues (k,) ascending incl. PlusI and eigenvectors (n, k)."""
from __future__ import annotations

from ...solvers.cdm import cdm
from ...spectrum import estimate_spectrum_bound


def OOC2_KrylovAv_A_EstimateSpectrumBound(KrylovAv, A, User_Seed=0):
    """(min, max) Ritz values of a 300-step Lanczos run on A (T1.py:135-192); the
    KrylovAv argument is accepted for signature compatibility, the product is the
    package's SpMM on the store A."""
    return estimate_spectrum_bound(A, steps=300, seed=User_Seed)


def S_HeigvalCDSIHD_HeigvecCDSIHD(A, A_diag, k=16, tol=1e-10, maxiter=1000000, User_WorkspaceSizeFactor=2,
                                  User_ChebyshevDegree=80, User_HalfMemMode=True, User_SpectrumBound=None,
                                  User_Q_HotellingDeflation=None, User_HotellingShift=10.0, User_Precision="f64",
                                  User_Block=1, User_Seed=0):
    assert User_SpectrumBound is not None, "ABORTED. The spectrum bound has to be initiated."
    assert User_WorkspaceSizeFactor > 1, "ABORTED. We require User_WorkspaceSizeFactor > 1 "
    assert User_Q_HotellingDeflation is None, ("ABORTED. We do not support Hotelling at the moment (Actually we "
                                               "do not need it if we have a mid-pass filter.) ")
    print("WARNING. Hotelling deflation not in use")
    return cdm(A, k=k, tol=tol, maxiter=maxiter, workspace_factor=User_WorkspaceSizeFactor,
               degree=User_ChebyshevDegree, spectrum_bound=User_SpectrumBound, precision=User_Precision,
               block=User_Block, seed=User_Seed)
