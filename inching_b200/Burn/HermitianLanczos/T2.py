"""Drop-in for InchingLiteInteger.Burn.HermitianLanczos.T2 (HermitianLanczos/T2.py:30-101)."""
from ...spectrum import estimate_spectrum_bound


def A_Adiag_EstimateSpectrumBound(A, A_diag, User_HalfMemMode=True, User_Steps=300, User_Seed=0,
                                  User_ReturnRitz=False):
    """(min, max) of the spectrum of A from a 300-step Lanczos run (2-tuple, as
    shipped).  User_ReturnRitz=True adds the Ritz values as a third element, the
    form the many-mode notebook indexes (its driver cell, lines 182-188)."""
    return estimate_spectrum_bound(A, steps=User_Steps, seed=User_Seed, return_ritz=User_ReturnRitz)
