"""Drop-in for InchingLiteInteger.Burn.PolynomialFilters.T0 (filter design, host)."""
from ...polyfilter import (PolParams, OOC0_OptimizePolynomialParamsOnDegree, balance_root as rootchb,  # noqa: F401
                           cheb_eval as ChebIv, damping_kernel)


def OOC1_DegreeM_DampingKernel(m, User_MaximumDegree=1000, User_DampingKernel="Jackson", dtype_temp=None):
    return damping_kernel(m, User_MaximumDegree, User_DampingKernel)
