"""Oracle eigensolvers: numpy restatements of the reference's TRLM, JDM (with
its projected GMRES), IRLM, Chebyshev-Davidson (CDM), Chebyshev filter
application and spectrum bound.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).  Every solver takes a
callable ``op(v) -> H v`` for the (+PlusI) Hessian so it can run on the scipy
half store of :mod:`oracle.hessian`.  Random start vectors come from a seeded
numpy generator (the reference uses CuPy's global RNG seeded 0), so outputs are
compared by eigenvalue / subspace / residual, never by bits.
"""
from __future__ import annotations

import numpy as np


def _deflated(op, Q, shift):
    if Q is None:
        return op
    return lambda v: op(v) + shift * (Q.T @ (Q @ v))


# ---------------------------------------------------------------------------
# Chebyshev filter application, Burn/PolynomialFilters/T2.py:28-92
# ---------------------------------------------------------------------------
def chebyshev_av(op, v, mu, cc, dd, m):
    vkm1 = np.zeros_like(v)
    vk = v.copy()
    y = v * mu[0]
    for k in range(1, m + 1):
        scal = 1.0 / dd if k == 1 else 2.0 / dd
        vkp1 = scal * (op(vk) - cc * vk) - (vkm1 if k > 1 else 0.0)
        y = y + mu[k] * vkp1
        vkm1, vk = vk, vkp1
    return y


# ---------------------------------------------------------------------------
# Spectrum bound, Burn/HermitianLanczos/T2.py:30-101 (300 Lanczos steps, no reorth)
# ---------------------------------------------------------------------------
def spectrum_bound(op, n, steps=300, seed=0):
    rng = np.random.default_rng(seed)
    alpha = np.zeros(steps + 1)
    beta = np.zeros(steps)
    v = rng.random(n) - 0.5
    v /= np.linalg.norm(v)
    f = op(v)
    a = v @ f
    f -= a * v
    alpha[0] = a
    for i in range(steps):
        b = np.linalg.norm(f)
        v0 = v
        v = f / b
        f = op(v) - b * v0
        a = f @ v
        f -= a * v
        alpha[i + 1] += a
        beta[i] += b
    T = np.diag(alpha) + np.diag(beta, -1) + np.diag(beta, 1)
    w = np.linalg.eigvalsh(T)
    return w.min(), w.max()


# ---------------------------------------------------------------------------
# TRLM, Burn/ThickRestartLanczosHotellingDeflation/T1.py:60-351,371-522
# ---------------------------------------------------------------------------
def _trd_eig(alpha, beta, beta_k, k, filtered):
    t = np.diag(alpha) + np.diag(beta[:-1], 1) + np.diag(beta[:-1], -1)
    if beta_k is not None:
        t[k, :k] = beta_k
        t[:k, k] = beta_k
    S, W = np.linalg.eigh(t)
    if not filtered:
        idx = np.argsort(S)[::-1]
        sel = idx[-k:][::-1]
    else:
        idx = np.argsort(S)
        sel = idx[-k:][::-1]
    return S[sel], W[:, sel]


def _lanczos(apply, V, u, alpha, beta, i_start, i_end):
    v = V[i_start].copy()
    for i in range(i_start, i_end):
        u[:] = apply(v)
        alpha[i] = v @ u
        uu = V[:i + 1] @ u
        u -= V[:i + 1].T @ uu
        beta[i] = np.linalg.norm(u)
        uu = V[:i + 1] @ u
        u -= V[:i + 1].T @ uu
        if i >= i_end - 1:
            break
        v = u / beta[i]
        V[i + 1] = v


def trlm(op, n, k=32, maxiter=10000, tol=0.0, workspace_factor=2, Q=None, shift=10.0,
         cheb=None, seed=0):
    """Returns (eigenvalues ascending incl. PlusI, eigenvectors (n, k), iterations)."""
    ncv = min(max(workspace_factor * k, k + 32), n - 1)
    if tol == 0:
        tol = np.finfo(np.float64).eps
    rng = np.random.default_rng(seed)
    alpha = np.zeros(ncv)
    beta = np.zeros(ncv)
    V = np.empty((ncv, n))
    u = rng.random(n)
    V[0] = u / np.linalg.norm(u)
    base = _deflated(op, Q, shift)
    if cheb is None:
        apply = base
    else:
        # filter first, deflation after (TRLM T1.py:441-458)
        apply = lambda v: chebyshev_av(op, v, *cheb) + (0 if Q is None else shift * (Q.T @ (Q @ v)))
    _lanczos(apply, V, u, alpha, beta, 0, ncv)
    S, W = _trd_eig(alpha, beta, None, k, cheb is not None)
    V[:k] = W.T @ V
    beta_k = beta[-1] * W[-1, :]
    res = np.linalg.norm(beta_k)
    it = 0
    for it in range(maxiter):
        beta[:k] = 0
        alpha[:k] = S
        u = u - V[:k].T @ (V[:k] @ u)
        u /= np.linalg.norm(u)
        V[k] = u
        u = apply(V[k])
        alpha[k] = V[k] @ u
        u -= alpha[k] * V[k]
        u -= V[:k].T @ beta_k
        beta[k] = np.linalg.norm(u)
        V[k + 1] = u / beta[k]
        _lanczos(apply, V, u, alpha, beta, k + 1, ncv)
        S, W = _trd_eig(alpha, beta, beta_k, k, cheb is not None)
        V[:k] = W.T @ V
        beta_k = beta[-1] * W[-1, :]
        res = np.linalg.norm(beta_k)
        if res <= tol:
            break
    if cheb is not None:
        S = np.array([V[i] @ op(V[i]) for i in range(k)])
    idx = np.argsort(S)
    return S[idx], V[idx].T.copy(), it


# ---------------------------------------------------------------------------
# JDM, Burn/JacobiDavidsonHotellingDeflation/T1.py:382-757 and the projected
# GMRES of IterativeSolvers.py:216-305
# ---------------------------------------------------------------------------
def gmres_deflate(matvec, b, x0, uu, tol, restart=20, maxiter=20):
    """Right-hand-side projected GMRES(restart) as in IterativeSolvers.py:216-305,
    including its observable quirks: the Arnoldi output is projected with
    (uu . z) (already ~0) and the routine returns the projected iterate ``mx``."""
    n = b.shape[0]
    x = x0.copy()
    b_norm = np.linalg.norm(b)
    if b_norm == 0:
        return b
    atol = tol * b_norm
    restart = min(restart, n)
    V = np.empty((n, restart))
    H = np.zeros((restart + 1, restart))
    e = np.zeros(restart + 1)
    iters = 0
    while True:
        mx = x.copy()
        mx -= (uu @ mx) * uu
        ax = matvec(mx)
        ax -= (uu @ ax) * uu
        r = b - ax
        r_norm = np.linalg.norm(r)
        if r_norm <= atol or iters >= maxiter:
            break
        v = r / r_norm
        V[:, 0] = v
        e[0] = r_norm
        for j in range(restart):
            z = v.copy()
            z -= (uu @ z) * uu
            u = matvec(z)
            u -= (uu @ z) * uu
            h = V[:, :j + 1].T @ u
            u -= V[:, :j + 1] @ h
            H[:j + 1, j] = h
            H[j + 1, j] = np.linalg.norm(u)
            if j + 1 < restart:
                v = u / H[j + 1, j]
                V[:, j + 1] = v
        y = np.linalg.lstsq(H, e, rcond=None)[0]
        x += V @ y
        iters += restart
    return mx


def jdm(op, n, k=16, tol=1e-10, maxiter=1000, correction_maxiter=20, workspace_factor=2,
        intermediate_tol=1e-3, gap=0.1, factoring_tol=1e-4, Q=None, shift=10.0, seed=0, time_budget=None):
    """Returns (eigenvalues ascending, eigenvectors (n, k), iterations, converged).
    With time_budget (s) the iteration stops early and returns what it has."""
    import time as _time
    t_start = _time.perf_counter()
    rng = np.random.default_rng(seed)
    jmax = k * workspace_factor
    jmin = min(n, k)
    Hop = _deflated(op, Q, shift)
    V = np.zeros((n, jmax + 1))
    Qc = np.zeros((n, jmin))
    eig = np.zeros(k)
    v0 = rng.random((n, 1)) - 0.5
    v0 /= np.sqrt((v0 * v0).sum(axis=0))
    Av = Hop(v0[:, 0])
    V[:, 0] = v0[:, 0]
    G = v0.T @ Av[:, None]
    theta = G[0, 0]
    nconv = 0
    jacc = 0
    jcur = 1
    for it in range(maxiter):
        if time_budget is not None and _time.perf_counter() - t_start > time_budget:
            idx = np.argsort(eig[:max(nconv, 1)])
            return eig[idx], Qc[:, idx], it, False
        S, W = np.linalg.eigh(G, UPLO="L")
        while True:
            theta = S[0]
            u = V[:, :W.shape[0]] @ W[:, :1]
            r = Hop(u[:, 0])[:, None] - theta * u
            cur = np.linalg.norm(r)
            sigma = theta - gap
            Qc[:, jacc] = u[:, 0]
            jcur = W.shape[0]
            if cur > tol or (nconv != k - 1 and len(S) <= 1):
                break
            eig[nconv] = theta
            nconv += 1
            jacc += 1
            V[:, :W.shape[1] - 1] = V[:, :W.shape[0]] @ W[:, 1:]
            jcur = W.shape[1] - 1
            S = S[1:]
            G, W = np.diag(S), np.identity(S.shape[0])
            if nconv == k:
                idx = np.argsort(eig)
                return eig[idx], Qc[:, idx], it, True
        if S.shape[0] == jmax:
            V[:, :jmin] = V[:, :W.shape[0]] @ W[:, :jmin]
            jcur = jmin
            S = S[:jmin]
            G, W = np.diag(S), np.identity(S.shape[0])
        sh = theta if cur < intermediate_tol else sigma
        matvec = lambda x, sh=sh: Hop(x) - sh * x
        uu = u[:, 0] / np.linalg.norm(u[:, 0])
        x0 = rng.random(n) * (cur * factoring_tol / n)
        z = gmres_deflate(matvec, -r[:, 0], x0, uu, cur * factoring_tol, 20, correction_maxiter)
        z = z[:, None]
        for i in range(jacc + 1):                     # MGS vs Q (T2.py:131-137)
            z = z - (z.T @ Qc[:, i:i + 1]) * Qc[:, i:i + 1]
        Vc = V[:, :jcur]                              # ICGS vs V (T2.py:98-117)
        r_pre = np.sqrt(abs(z.T @ z))
        for _ in range(3):
            z = z - Vc @ (Vc.T @ z)
            r1 = np.sqrt(abs(z.T @ z))
            if r1 > r_pre / 2:
                break
            r_pre = r1
        z = z / r1
        Az = Hop(z[:, 0])[:, None]
        G = np.vstack((np.hstack((G, Vc.T @ Az)), np.hstack((Az.T @ Vc, Az.T @ z))))
        V[:, jcur] = z[:, 0]
    eig[nconv] = theta
    nconv += 1
    idx = np.argsort(eig)
    return eig[idx], Qc[:, idx], maxiter, False


def ritz_residuals(op, lam, vecs):
    """||H v - lambda v||_2 per column."""
    return np.array([np.linalg.norm(op(vecs[:, i]) - lam[i] * vecs[:, i]) for i in range(len(lam))])


# ---------------------------------------------------------------------------
# Chebyshev-Davidson, Burn/ChebyshevDavidsonSubspaceIteration/T1.py:229-623
# ---------------------------------------------------------------------------
def cdm_filter(op, x, degree, low, high):
    """Unscaled Chebyshev filter T_{degree+1}((c - H)/e) x on [low, high]
    (T1.py:195-226): y = (c x - H x)/e, then degree times y' = 2 (c y - H y)/e - x."""
    e = (high - low) / 2.0
    c = (high + low) / 2.0
    z = x.copy()
    y = (c * z - op(z)) / e
    for _ in range(degree):
        ynew = 2.0 * (c * y - op(y)) / e - z
        z, y = y, ynew
    return y


def cdm(op, n, k=16, tol=1e-10, maxiter=100000, workspace_factor=2, degree=80, spectrum_bound=None, seed=0):
    """Single-vector Chebyshev-Davidson as in T1.py:229-623: one filtered vector
    per outer step, classical + modified Gram-Schmidt, Rayleigh-Ritz over the
    active (unconverged) columns, restart when the workspace is full, convergence
    of the first active Ritz pair at tol * max|theta|, lower filter bound moved
    to the median active Ritz value.  After a convergence the next filter input is
    the just-converged column, as the reference does (T1.py:596-597).
    Returns (eigenvalues ascending, eigenvectors (n, k), iterations, converged)."""
    assert spectrum_bound is not None, "ABORTED. The spectrum bound has to be initiated."
    assert workspace_factor > 1, "ABORTED. We require User_WorkspaceSizeFactor > 1 "
    rng = np.random.default_rng(seed)
    jmin = min(n, k)
    jmax = workspace_factor * jmin
    V = np.zeros((n, jmax))
    AV = np.zeros((n, jmax))
    G = np.zeros((jmax, jmax))
    conv = np.zeros(jmin + 1)
    thb = spectrum_bound[-1] + 1e-5
    x = rng.random(n)
    x /= np.linalg.norm(x)
    V[:, 0] = x
    AV[:, 0] = op(x)
    G[0, 0] = x @ AV[:, 0]
    squeeze = (thb + G[0, 0]) / 2.0
    beta = max(1e-14, abs(G[0, 0]))
    tolr = tol * beta
    nc, nc1, j = 0, 1, 1
    for it in range(maxiter):
        v = cdm_filter(op, x, degree, squeeze, thb)
        v /= np.linalg.norm(v)
        for _ in range(2):                           # ICGS against the whole basis
            v -= V[:, :j] @ (V[:, :j].T @ v)
        v /= np.linalg.norm(v)
        for i in range(nc):                          # MGS against converged columns
            v -= (V[:, i] @ v) * V[:, i]
        V[:, j] = v
        AV[:, j] = op(v)
        r = V[:, nc:j + 1].T @ AV[:, j]
        G[j, nc:j] = r[:-1]
        G[nc:j + 1, j] = r
        G = 0.5 * (G + G.T)
        S, W = np.linalg.eigh(G[nc:j + 1, nc:j + 1])
        if j + 1 >= jmax:
            jr = max(nc1, jmin + 5, min(jmin + nc, jmax - 5))
        else:
            jr = j + 1
        nn = jr - nc
        V[:, nc:jr] = V[:, nc:j + 1] @ W[:, :nn]
        AV[:, nc:jr] = AV[:, nc:j + 1] @ W[:, :nn]
        G[nc:jr, nc:jr] = np.diag(S[:nn])
        beta = max(beta, np.max(np.abs(S)))
        tolr = tol * beta
        theta = S[0]
        x = V[:, nc].copy()
        res = np.linalg.norm(AV[:, nc] - theta * x)
        if res < tolr:
            conv[nc] = theta
            nc += 1
            nc1 = nc + 1
            if nc >= jmin:
                lam = conv[:-1]
                idx = np.argsort(lam)
                return lam[idx], V[:, idx], it + 1, True
            x = V[:, nc - 1].copy()
        j = jr
        squeeze = max(float(np.median(S)), spectrum_bound[0])
    lam = conv[:-1]
    idx = np.argsort(lam)
    return lam[idx], V[:, idx], maxiter, False
