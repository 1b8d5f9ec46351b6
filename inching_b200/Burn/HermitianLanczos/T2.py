"""Drop-in for InchingLiteInteger.Burn.HermitianLanczos.T2 (HermitianLanczos/T2.py:30-101)."""
from ...spectrum import estimate_spectrum_bound


def A_Adiag_EstimateSpectrumBound(A, A_diag, User_HalfMemMode=True, User_Steps=300, User_Seed=0):
    """(min, max) of the spectrum of A from a 300-step Lanczos run (2-tuple, as shipped)."""
    return estimate_spectrum_bound(A, steps=User_Steps, seed=User_Seed)
