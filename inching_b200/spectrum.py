"""Spectrum bounds, kernel-polynomial (KPM) eigenvalue counts and the filter
window search, on the GPU.

Reference counterparts:
  * A_Adiag_EstimateSpectrumBound           Burn/HermitianLanczos/T2.py:30-101
    (300 Lanczos steps without reorthogonalisation, extremal Ritz values)
  * A_Adiag_PolynomialParams_KpmEstimate     Burn/PolynomialFilters/T2.py:96-138
    (stochastic trace of the filter: one ChebyshevAv per random probe)
  * A_Adiag_OptimizePolynomialParamsOnMemory Burn/PolynomialFilters/T2.py:142-255
    (bisection of the window's right edge until the KPM count is within a margin)
Here all KPM probes of one estimate run as ONE block: the Chebyshev recurrence
is applied to an (n, trials) multivector with the fused SpMM, and the per-probe
density terms are column dot products.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import polyfilter
from .krylov import HessianOperator


def estimate_spectrum_bound(A, steps=300, seed=0, precision="f64", return_ritz=False):
    """(min, max) Ritz values of a `steps`-step Lanczos run from a random start
    (with return_ritz, also all Ritz values, ascending)."""
    dev = A.device
    N = A.shape[0]
    op = HessianOperator(A, prec=32 if precision == "mixed" else 64)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    v = torch.rand(N, generator=g, dtype=torch.float64, device=dev) - 0.5
    v /= torch.linalg.vector_norm(v)
    alpha = torch.zeros(steps + 1, dtype=torch.float64, device=dev)
    beta = torch.zeros(steps, dtype=torch.float64, device=dev)
    f = op(v)
    a = torch.dot(v, f)
    f -= a * v
    alpha[0] = a
    v0 = torch.empty_like(v)
    for i in range(steps):
        b = torch.linalg.vector_norm(f)
        v0.copy_(v)
        torch.div(f, b, out=v)
        op(v, out=f)
        f -= b * v0
        a = torch.dot(f, v)
        f -= a * v
        alpha[i + 1] = a
        beta[i] = b
    al = alpha.cpu().numpy()
    be = beta.cpu().numpy()
    T = np.diag(al) + np.diag(be, -1) + np.diag(be, 1)
    w = np.linalg.eigvalsh(T)
    if return_ritz:
        return float(w.min()), float(w.max()), w
    return float(w.min()), float(w.max())


def kpm_rho(A, params, trials=1000, seed=0, precision="f64", batch=256):
    """Per-probe KPM density terms rho_t (ChebyshevAv(..., User_ReturnRho=True))."""
    dev = A.device
    N = A.shape[0]
    prec = 32 if precision == "mixed" else 64
    dt = torch.float64 if prec == 64 else torch.float32
    p = params
    m = int(p.AdjustedDegree)
    cc, dd = float(p.cc), float(p.dd)
    jac = np.asarray(p.AdjustedDampingKernels, dtype=np.float64)
    ta, tb = float(p.theta_a), float(p.theta_b)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    out = []
    for t0 in range(0, trials, batch):
        T = min(batch, trials - t0)
        v = torch.randn((N, T), generator=g, dtype=torch.float64, device=dev)
        v /= torch.linalg.vector_norm(v, dim=0, keepdim=True)
        rho = torch.full((T,), ta - tb, dtype=torch.float64, device=dev)
        vk = v.to(dt).clone()          # never alias the probes
        vkm1 = torch.empty_like(vk)
        for k in range(1, m + 1):
            scal = 1.0 / dd if k == 1 else 2.0 / dd
            if k == 1:
                A.matmul(vk, out=vkm1, prec=prec, alpha=scal, gamma=-scal * cc)
            else:
                A.matmul(vk, out=vkm1, prec=prec, alpha=scal, gamma=-scal * cc, beta=-1.0, Yin=vkm1)
            vk, vkm1 = vkm1, vk
            dots = (vk.double() * v).sum(dim=0)
            rho -= 2 * jac[k] * dots * (math.sin(k * tb) - math.sin(k * ta)) / k
        out.append(rho / math.pi)
    return torch.cat(out)


def kpm_count(A, params, trials=1000, seed=0, precision="f64"):
    """Estimated number of eigenvalues in the filter window, int(mean rho * N) + 1."""
    rho = kpm_rho(A, params, trials, seed, precision)
    return int(float(rho.mean()) * A.shape[0]) + 1


def optimize_params_on_memory(A, User_MaximumDegree=1000, User_MinimumDegree=10, User_DampingKernel="Jackson",
                              User_ExtremalIntervalDefinition=1e-10, User_WantedInterval=(36.8, 37.2),
                              User_SpectrumBound=(1.0, 759.0), User_DesignatedStart=None,
                              User_WantedNumberEigenvalue=12, User_AffordableMemoryMargin=5,
                              User_NumberKpmTrials=1000, User_ConvergenceRatio=0.1, precision="f64", seed=0):
    """Bisection on the right edge of the window (PolynomialFilters/T2.py:142-255)."""
    design = lambda lo_hi: polyfilter.OOC0_OptimizePolynomialParamsOnDegree(
        User_MaximumDegree=User_MaximumDegree, User_MinimumDegree=User_MinimumDegree,
        User_DampingKernel=User_DampingKernel, User_ExtremalIntervalDefinition=User_ExtremalIntervalDefinition,
        User_WantedInterval=lo_hi, User_SpectrumBound=User_SpectrumBound, User_ConvergenceRatio=User_ConvergenceRatio)
    count = lambda pol: kpm_count(A, pol, User_NumberKpmTrials, seed, precision)
    window = [User_WantedInterval[0], User_SpectrumBound[1]]
    if User_DesignatedStart is not None:
        pol = design((User_WantedInterval[0], User_DesignatedStart))
        if count(pol) > User_WantedNumberEigenvalue * 2:
            window = [User_WantedInterval[0], User_DesignatedStart]
    left, right = window
    pol, cnt = None, None
    while right - left >= 1e-8:
        mid = (left + right) / 2
        window[1] = mid
        pol = design(tuple(window))
        cnt = count(pol)
        if abs(cnt - User_WantedNumberEigenvalue) <= User_AffordableMemoryMargin:
            break
        if cnt < User_WantedNumberEigenvalue:
            left = mid
        else:
            right = mid
    return pol, cnt, tuple(window)
