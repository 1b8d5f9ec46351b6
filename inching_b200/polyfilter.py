"""Chebyshev polynomial filter design (host, FP64).

Restates the filter construction of InchingLiteInteger/Burn/PolynomialFilters/T0.py,
which follows EVSL (Li, Xi, Vecharynski, Yang, Saad, SIAM J. Sci. Comput. 38 (2016)):
  * damping kernels (Jackson / Lanczos sigma / none)           T0.py:25-55
  * extremal interval: scaled-and-shifted Chebyshev "base filter" whose degree is
    the first one with value < 0.1 at the interval edge         T0.py:64-169
  * interior interval: Dirac-delta-type expansion centred by a Newton/bisection
    balancing step so both interval edges get the same value, degree grown until
    both edges are below ConvergenceRatio * centre value         T0.py:182-303
  * interval normalisation to [-1, 1] by cc, dd                T0.py:313-392
The returned PolParams object carries the same attributes the reference's does
(AdjustedCoefficients, AdjustedDegree, AdjustedDampingKernels, cc, dd, theta_a,
theta_b, gam, ...), so it can be passed wherever User_PolynomialParams is taken.
"""
from __future__ import annotations

import math

import numpy as np


class PolParams:
    def __init__(self, User_MaximumDegree=10000, User_MinimumDegree=2, User_DampingKernel="Jackson", mu=None,
                 deg=0, User_ExtremalIntervalDefinition=1e-9, User_ConvergenceRatio=0.1):
        self.User_MaximumDegree = User_MaximumDegree
        self.User_MinimumDegree = User_MinimumDegree
        self.User_DampingKernel = User_DampingKernel
        self.User_ExtremalIntervalDefinition = User_ExtremalIntervalDefinition
        self.User_ConvergenceRatio = User_ConvergenceRatio
        self.AdjustedCoefficients = mu
        self.AdjustedDampingKernels = None
        self.AdjustedDegree = deg


def damping_kernel(m, size, kind="Jackson"):
    """Damping factors g_k, k = 0..m (array of length size+1, g_0 = 1/2)."""
    g = np.zeros(size + 1, dtype=np.float64)
    k = np.arange(1, m + 1, dtype=np.float64)
    if kind == "Jackson":
        t = np.pi / (m + 2)
        a1 = 1.0 / (m + 2)
        g[1:m + 1] = a1 * np.sin((k + 1) * t) / np.sin(t) + (1 - (k + 1) * a1) * np.cos(k * t)
    elif kind == "LanczosSigma":
        t = np.pi / (m + 1)
        g[1:m + 1] = np.sin(k * t) / (k * t)
    else:
        g[1:] = 1.0
    g[0] = 0.5
    return g


def _extremal(pol, a, b):
    """Base filter for an interval touching -1 or +1 (T0.py:64-169)."""
    maxdeg, mindeg = pol.User_MaximumDegree, pol.User_MinimumDegree
    gam = np.sign(b - (1 - pol.User_ExtremalIntervalDefinition))
    x = a if gam > 0 else b
    a, b = sorted([x - gam * 0.1 * np.sqrt((1 - gam * x) / 2), -1 * gam])
    c = (b + a) * 0.5
    e = (b - a) * 0.5
    sig = e / (gam - c)
    sig1 = sig
    # degree: first k >= mindeg with the scaled polynomial below 0.1 at x
    g0, g1 = 1.0, (x - c) * (sig1 / e)
    m = 1
    for k in range(2, maxdeg + 1):
        sn = 1.0 / (2.0 / sig1 - sig)
        gn = 2 * (x - c) * (sn / e) * g1 - (sig * sn) * g0
        g0, g1 = g1, gn
        sig = sn
        m += 1
        if (g1 < 0.1) and (k >= mindeg):
            break
    bar = g1
    # monomial-in-T coefficients of the same recurrence
    sig = e / (gam - c)
    tau = 2 / sig1
    c0 = np.zeros(maxdeg + 1)
    c1 = np.zeros(maxdeg + 1)
    cn = np.zeros(maxdeg + 1)
    c0[0] = 1.0
    c1[0] = -c * (sig1 / e)
    c1[1] = sig1 / e
    for k in range(2, m + 1):
        sn = 1.0 / (tau - sig)
        s1 = sn / e
        cn[:k] = c1[1:k + 1]
        cn[1] += c1[0]
        cn[1:k + 1] += c1[:k]
        cn *= s1
        cn[:k + 1] -= (2 * s1 * c) * c1[:k + 1]
        cn[:k + 1] -= (sig * sn) * c0[:k + 1]
        c0[:k + 1] = c1[:k + 1]
        c1[:k + 1] = cn[:k + 1]
        sig = sn
    pol.AdjustedCoefficients = c1[:m + 1] * pol.AdjustedDampingKernels[:m + 1]
    pol.AdjustedDegree = m
    pol.bar = bar
    pol.gam = gam
    return pol


def _cheb_sum_at(v, thc, jac):
    return np.sum(v * np.cos(np.arange(jac.shape[0]) * thc) * jac)


def balance_root(m, v, jac, tha, thb):
    """Newton steps safeguarded by bisection for the centre angle at which the
    damped delta expansion takes equal values at both edges (T0.py:182-226)."""
    tol = abs(tha - thb) * 1e-6
    thc = (tha + thb) / 2
    ks = np.arange(1, m + 1, dtype=np.float64)
    for _ in range(759):
        f = _cheb_sum_at(v, thc, jac)
        d = np.sum(jac[1:m + 1] * ks * np.sin(np.arange(1, m + 1) * thc) * v[1:m + 1])
        thn = thc + f / d
        if abs(f) < tol or abs(thc - thn) < np.finfo(np.float64).eps * abs(thc):
            break
        if f > 0:
            if thn < thb or thn > tha:
                thn = 0.5 * (thc + tha)
            thb = thc
        else:
            if thn < thb or thn > tha:
                thn = 0.5 * (thc + thb)
            tha = thc
        thc = thn
    return np.cos(np.arange(jac.shape[0]) * thc) * jac, thc


def cheb_eval(m, mu, xi):
    """sum_k mu_k T_k(xi) by the three-term recurrence (T0.py:229-245)."""
    xi = np.asarray(xi, dtype=np.float64)
    tkm1 = np.zeros_like(xi)
    tk = np.ones_like(xi)
    y = tk * mu[0]
    for k in range(1, m + 1):
        s = 1.0 if k == 1 else 2.0
        tkp1 = s * xi * tk - tkm1
        y = y + mu[k] * tkp1
        tkm1, tk = tk, tkp1
    return y


def _interior(pol, aa, bb):
    """Balanced interior filter (T0.py:248-303)."""
    thb = np.arccos(bb)
    tha = np.arccos(aa)
    maxdeg, mindeg = pol.User_MaximumDegree, pol.User_MinimumDegree
    v = np.zeros(maxdeg + 1)
    v[:mindeg] = np.cos(np.arange(mindeg) * thb) - np.cos(np.arange(mindeg) * tha)
    mu = None
    gam = None
    m = mindeg
    for m in range(mindeg, maxdeg):
        v[m] = np.cos(m * thb) - np.cos(m * tha)
        jac = damping_kernel(m, maxdeg, pol.User_DampingKernel)
        new_mu, thc = balance_root(m, v, jac, tha, thb)
        gam = np.cos(thc)
        t = cheb_eval(m, new_mu, np.array([gam]))
        vals = cheb_eval(m, new_mu, np.array([aa, bb]))
        mu = new_mu / t
        if np.all(vals <= t * pol.User_ConvergenceRatio):
            m += 1
            break
    pol.gam = gam
    pol.AdjustedDegree = m - 1
    pol.AdjustedCoefficients = mu
    return pol


def OOC0_OptimizePolynomialParamsOnDegree(User_MaximumDegree=1000, User_MinimumDegree=10,
                                          User_DampingKernel="Jackson", User_ExtremalIntervalDefinition=1e-9,
                                          User_WantedInterval=(36.8, 37.2), User_SpectrumBound=(1.0, 759.0),
                                          User_ConvergenceRatio=0.1):
    """Filter for the wanted interval inside the spectrum bound (T0.py:313-392)."""
    pol = PolParams(User_MaximumDegree=User_MaximumDegree, User_MinimumDegree=User_MinimumDegree,
                    User_DampingKernel=User_DampingKernel,
                    User_ExtremalIntervalDefinition=User_ExtremalIntervalDefinition,
                    User_ConvergenceRatio=User_ConvergenceRatio)
    eps = User_ExtremalIntervalDefinition
    aa = max(User_WantedInterval[0], User_SpectrumBound[0])
    bb = min(User_WantedInterval[1], User_SpectrumBound[1])
    cc = 0.5 * (User_SpectrumBound[1] + User_SpectrumBound[0])
    dd = 0.5 * (User_SpectrumBound[1] - User_SpectrumBound[0])
    aa = max((aa - cc) / dd, -1.0)
    bb = min((bb - cc) / dd, 1.0)
    if aa <= -1.0 + eps:
        aa = -1.0
    if bb >= 1.0 - eps:
        bb = 1.0
    assert not ((aa <= -1.0 + eps) & (bb >= 1.0 - eps)), \
        "ABORTED. Too greedy! Both ends of the wanted interval are close to the extremal. relax either side"
    pol.theta_a = np.arccos(aa)
    pol.theta_b = np.arccos(bb)
    pol.cc = cc
    pol.dd = dd
    pol.AdjustedDampingKernels = damping_kernel(pol.User_MaximumDegree, pol.User_MaximumDegree + 1,
                                                pol.User_DampingKernel)
    if (aa <= -1.0 + eps) or (bb >= 1.0 - eps):
        pol = _extremal(pol, aa, bb)
    else:
        pol = _interior(pol, aa, bb)
    pol.User_WantedInterval = User_WantedInterval
    pol.User_SpetrumBound = User_SpectrumBound
    return pol
