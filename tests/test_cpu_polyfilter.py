"""Chebyshev filter design against the reference's own outputs: the fixture holds
OOC0_OptimizePolynomialParamsOnDegree of the reference
(InchingLiteInteger/Burn/PolynomialFilters/T0.py), run by tests/golden/make_golden.py
on 4 windows (2 extremal, 2 interior) x convergence ratio 0.1 / 0.7 x Jackson /
Lanczos-sigma kernels.  The package's design, called directly and through the
drop-in module path, must reproduce degree, coefficients and the scalars (c, d,
theta_a, theta_b, gamma) bit for bit."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

FIX = np.load(os.path.join(GOLDEN, "polyfilter.npz"))
KEYS = sorted({k.rsplit("_", 1)[0] for k in FIX.files if k.startswith("w")})


def test_fixture_covers_sixteen_designs():
    assert len(KEYS) == 16


@pytest.mark.parametrize("key", KEYS)
def test_filter_design_bit_identical_to_reference(key):
    from inching_b200 import polyfilter
    from inching_b200.Burn.PolynomialFilters import T0
    lo, hi, blo, bhi, conv, max_deg, min_deg = FIX[key + "_args"]
    kern = str(FIX[key + "_kernel"])
    kw = dict(User_WantedInterval=(lo, hi), User_SpectrumBound=(blo, bhi), User_MaximumDegree=int(max_deg),
              User_MinimumDegree=int(min_deg), User_DampingKernel=kern, User_ExtremalIntervalDefinition=1e-9,
              User_ConvergenceRatio=float(conv))
    for design in (polyfilter.OOC0_OptimizePolynomialParamsOnDegree, T0.OOC0_OptimizePolynomialParamsOnDegree):
        pol = design(**kw)
        assert int(pol.AdjustedDegree) == int(FIX[key + "_deg"])
        mu = np.asarray(pol.AdjustedCoefficients, np.float64)
        assert mu.shape == FIX[key + "_mu"].shape and np.array_equal(mu, FIX[key + "_mu"])
        scal = np.array([pol.cc, pol.dd, pol.theta_a, pol.theta_b, float(pol.gam)], np.float64)
        assert np.array_equal(scal, FIX[key + "_scal"])
