"""Drop-in for InchingLiteInteger.Burn.PolynomialFilters.T2: Chebyshev filter
application, KPM eigenvalue counts and the window search (T2.py:16-255)."""
from __future__ import annotations

import torch

from ...krylov import ChebyshevFilter
from ...spectrum import kpm_count, optimize_params_on_memory


class OOC2_A_Adiag_ChebyshevAv:
    def __init__(self, A, A_diag, User_PolynomialParams=None, User_HalfMemMode=True, User_Precision="f64"):
        assert User_PolynomialParams is not None, "ABORTED. You must initiate with a found Polynomial Param"
        self.A = A
        self.User_PolynomialParams = User_PolynomialParams
        self._f = ChebyshevFilter(A, User_PolynomialParams, prec=32 if User_Precision == "mixed" else 64)

    def ChebyshevAv(self, A, v, User_ReturnRho=False):
        if User_ReturnRho:
            y, rho = self._f(v, return_rho=True)
            return y, rho
        return self._f(v)


def A_Adiag_PolynomialParams_KpmEstimate(A, A_diag, User_HalfMemMode=True, User_PolynomialParams=None,
                                         User_NumberKpmTrials=1000, User_Seed=0):
    assert User_PolynomialParams is not None, "ABORTED. You must initiate with a found Polynomial Param"
    return kpm_count(A, User_PolynomialParams, User_NumberKpmTrials, User_Seed)


def A_Adiag_OptimizePolynomialParamsOnMemory(A, A_diag, User_MaximumDegree=1000, User_MinimumDegree=10,
                                             User_DampingKernel="Jackson", User_ExtremalIntervalDefinition=1e-10,
                                             User_WantedInterval=(36.8, 37.2), User_SpectrumBound=(1.0, 759.0),
                                             User_DesignatedStart=None, User_WantedNumberEigenvalue=12,
                                             User_AffordableMemoryMargin=5, User_HalfMemMode=True,
                                             User_NumberKpmTrials=1000, User_ConvergenceRatio=0.1):
    return optimize_params_on_memory(
        A, User_MaximumDegree=User_MaximumDegree, User_MinimumDegree=User_MinimumDegree,
        User_DampingKernel=User_DampingKernel, User_ExtremalIntervalDefinition=User_ExtremalIntervalDefinition,
        User_WantedInterval=User_WantedInterval, User_SpectrumBound=User_SpectrumBound,
        User_DesignatedStart=User_DesignatedStart, User_WantedNumberEigenvalue=User_WantedNumberEigenvalue,
        User_AffordableMemoryMargin=User_AffordableMemoryMargin, User_NumberKpmTrials=User_NumberKpmTrials,
        User_ConvergenceRatio=User_ConvergenceRatio)
