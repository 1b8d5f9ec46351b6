"""CPU baseline of the hot path on the host cores.  TEST/MEASUREMENT
INFRASTRUCTURE ONLY: used by bench.py's cpu_baseline leg and its reference arm.

It runs the reference's algorithm on the CPU: neighbour lists with scipy's
cKDTree queried exactly as InchingLiteInteger/Fuel/Coordinate/T1.py:218-245
does (all host threads, workers=-1), the oracle's sequential Cuthill-McKee
(T1.py:254-323), the oracle's FP64 Hessian (Fuel/T1.py:276-455), the rigid-body
basis of the drivers and the oracle's Jacobi-Davidson (JDM T1.py:382-757) for a
bounded time.  The reference has no CPU eigensolver (its solvers need CuPy), so
this restatement is the CPU implementation that is timed.
"""
from __future__ import annotations

import os
import time

import numpy as np

from . import graph, hessian, solvers


def kdtree_neighbor_lists(X_nm, rc_gamma_A=8.0):
    from scipy.spatial import cKDTree
    tree = cKDTree(X_nm)
    nl = tree.query_ball_point(X_nm, rc_gamma_A / 10.0, p=2.0, eps=0, workers=-1, return_sorted=True)
    deg = np.fromiter((len(v) for v in nl), dtype=np.int32, count=len(nl))
    rowptr = np.zeros(len(nl) + 1, dtype=np.int64)
    rowptr[1:] = np.cumsum(deg)
    cols = np.concatenate([np.asarray(v, dtype=np.int32) for v in nl])
    return deg, rowptr, cols


def cpu_time_to_modes(X_nm, k, budget_s=15.0, tol_rel=1e-6, plain_iterations=None):
    """Preprocessing in full, then JDM for at most budget_s seconds.

    Returns a dict with the measured pieces and, when plain_iterations (outer
    JDM iterations the identical GPU algorithm needed for all k modes) is given,
    the projection t_pre + t_per_iteration * plain_iterations."""
    t0 = time.perf_counter()
    deg, rowptr, cols = kdtree_neighbor_lists(X_nm)
    order, undo = graph.cuthill_mckee(rowptr, cols, deg)
    Xr = X_nm[order]
    _, rp2, c2 = kdtree_neighbor_lists(Xr)
    A, Ad = hessian.hessian_lower(Xr, 8.0, 1.0, rowptr=rp2, cols=c2)
    Q = hessian.rigid_body_basis(Xr)
    t_pre = time.perf_counter() - t0
    AT = A.T.tocsr()
    op = lambda v: A @ v + AT @ v - Ad * v
    n = A.shape[0]
    normH = abs(A).sum(axis=1).max() * 2
    t1 = time.perf_counter()
    ev, _, iters, conv = solvers.jdm(op, n, k=k, tol=tol_rel * normH, Q=Q, shift=10.0, time_budget=budget_s)
    t_solve = time.perf_counter() - t1
    per_it = t_solve / max(iters, 1)
    out = dict(preprocess_s=t_pre, solve_sample_s=t_solve, sample_iterations=int(iters),
               seconds_per_iteration=per_it, converged_in_sample=bool(conv),
               cores=len(os.sched_getaffinity(0)))
    if plain_iterations is not None:
        out["projected_s"] = t_pre + per_it * plain_iterations
    return out


def arpack_time_to_modes(X_nm, k):
    """The reference's own CPU baseline (Command8A/commandArpack_Pdb_0064_EPYC.py:
    285-328): the Hessian's lower triangle symmetrised, then
    scipy.sparse.linalg.eigsh(A, k, which='SA') -- no deflation, so the k + 6
    lowest (six rigid-body modes at PlusI first).  Preprocessing as in
    cpu_time_to_modes.  Returns (seconds, eigenvalues of the k non-rigid modes)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as sla
    t0 = time.perf_counter()
    deg, rowptr, cols = kdtree_neighbor_lists(X_nm)
    order, _ = graph.cuthill_mckee(rowptr, cols, deg)
    Xr = X_nm[order]
    _, rp2, c2 = kdtree_neighbor_lists(Xr)
    A, _ = hessian.hessian_lower(Xr, 8.0, 1.0, rowptr=rp2, cols=c2)
    A_sym = (A + sp.tril(A, k=-1).T).tocsr()
    w = sla.eigsh(A_sym, k=k + 6, which="SA", return_eigenvectors=False)
    return time.perf_counter() - t0, np.sort(w)[6:]
