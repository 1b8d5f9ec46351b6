"""Drop-in for InchingLiteInteger.Burn.JacobiDavidsonHotellingDeflation.T1 (JDM,
T1.py:382-757).  Returns torch CUDA tensors: eigenvalues (k,) ascending incl.
PlusI and eigenvectors (n, k)."""
from __future__ import annotations

from ...solvers.jdm import jdm


def S_HeigvalJDMHD_HeigvecJDMHD(A, A_diag, k=16, tol=1e-10, maxiter=1000, User_CorrectionSolverMaxiter=20,
                                User_WorkspaceSizeFactor=2, User_HalfMemMode=True,
                                User_IntermediateConvergenceTol=1e-3, User_GapEstimate=0.1,
                                User_FactoringToleranceOnCorrection=1e-4, User_Q_HotellingDeflation=None,
                                User_HotellingShift=10.0, User_PolynomialParams=None, User_Precision="f64",
                                User_Seed=0):
    return jdm(A, k=k, tol=tol, maxiter=maxiter, correction_maxiter=User_CorrectionSolverMaxiter,
               workspace_factor=User_WorkspaceSizeFactor, intermediate_tol=User_IntermediateConvergenceTol,
               gap=User_GapEstimate, factoring_tol=User_FactoringToleranceOnCorrection,
               Q=User_Q_HotellingDeflation, shift=User_HotellingShift, polynomial=User_PolynomialParams,
               precision=User_Precision, seed=User_Seed)
