"""Oracle for the integer/graph part of the path: neighbour lists, degrees,
k-d-tree Cuthill-McKee order, row-batch heads and ungapped band slices.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).  Pure numpy / Python loops,
meant for inputs of up to a few 10^4 atoms.
"""
from __future__ import annotations

import numpy as np


def neighbor_lists(X_nm: np.ndarray, rc_gamma_A: float = 8.0, cell=None):
    """All j with |x_j - x_i| <= rc, self included, sorted ascending.

    Distance rule of scipy's cKDTree.query_ball_point (p=2, eps=0) as called by
    the reference (InchingLiteInteger/Fuel/Coordinate/T1.py:239,276): the squared
    distance is accumulated in axis order, ((dx*dx) + dy*dy) + dz*dz, each step
    rounded to double, and compared with r*r, r = rc_Gamma/10 (T1.py:209).
    Returns (degree int32 (N,), rowptr int64 (N+1,), cols int32 (nnz,)).
    """
    X = np.ascontiguousarray(X_nm, dtype=np.float64)
    n = X.shape[0]
    rc = rc_gamma_A / 10.0
    r2 = rc * rc
    if n == 0:
        return np.zeros(0, np.int32), np.zeros(1, np.int64), np.zeros(0, np.int32)
    lo = X.min(axis=0)
    cellsz = rc
    ci = np.floor((X - lo) / cellsz).astype(np.int64)
    dims = ci.max(axis=0) + 1
    key = (ci[:, 0] * dims[1] + ci[:, 1]) * dims[2] + ci[:, 2]
    srt = np.argsort(key, kind="stable")
    ks = key[srt]
    lists = []
    for i in range(n):
        c = ci[i]
        cand = []
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    cc = c + (dx, dy, dz)
                    if (cc < 0).any() or (cc >= dims).any():
                        continue
                    k = (cc[0] * dims[1] + cc[1]) * dims[2] + cc[2]
                    a = np.searchsorted(ks, k, "left")
                    b = np.searchsorted(ks, k, "right")
                    if b > a:
                        cand.append(srt[a:b])
        cand = np.concatenate(cand)
        d = X[cand] - X[i]
        s = d[:, 0] * d[:, 0]
        s = s + d[:, 1] * d[:, 1]
        s = s + d[:, 2] * d[:, 2]
        lists.append(np.sort(cand[s <= r2]).astype(np.int32))
    deg = np.array([len(v) for v in lists], dtype=np.int32)
    rowptr = np.zeros(n + 1, dtype=np.int64)
    rowptr[1:] = np.cumsum(deg)
    return deg, rowptr, np.concatenate(lists)


IMAGES_XY = ((0, 0), (1, 0), (-1, 0), (0, 1), (0, -1), (1, 1), (1, -1), (-1, 1), (-1, -1))


def neighbor_lists_pbc_xy(X_nm: np.ndarray, rc_gamma_A: float, box_xy):
    """Neighbour lists with periodic xy images, as X_cKDTreePbcXy.query_ball_point
    (InchingLiteInteger/Fuel/Coordinate/T1.py:67-161) builds them for a
    multi-point query: for each image shift s in the instruction order
    (T1.py:98-107) the query point is x_i + s (one rounding, numpy's
    xx + box * instr), the distance rule is cKDTree's, each image's list is sorted
    and the nine lists are concatenated.  The box sizes must exceed rc (T1.py:94-95).
    Returns (degree int32, rowptr int64, cols int32, image int8)."""
    X = np.ascontiguousarray(X_nm, dtype=np.float64)
    n = X.shape[0]
    rc = rc_gamma_A / 10.0
    bx, by = float(box_xy[0]), float(box_xy[1])
    assert bx > rc, "ABORTED. The PBC box size X is smaller than rc gamma."
    assert by > rc, "ABORTED. The PBC box size Y is smaller than rc gamma."
    r2 = rc * rc
    lists, imgs = [[] for _ in range(n)], [[] for _ in range(n)]
    for k, (ix, iy) in enumerate(IMAGES_XY):
        shift = np.array([bx * ix, by * iy, 0.0])
        Q = X + shift
        for a in range(0, n, 512):
            q = Q[a:a + 512]
            d = X[None, :, :] - q[:, None, :]
            s = d[..., 0] * d[..., 0]
            s = s + d[..., 1] * d[..., 1]
            s = s + d[..., 2] * d[..., 2]
            for r in range(q.shape[0]):
                js = np.nonzero(s[r] <= r2)[0].astype(np.int32)
                lists[a + r].append(js)
                imgs[a + r].append(np.full(len(js), k, np.int8))
    rows = [np.concatenate(v) for v in lists]
    deg = np.array([len(v) for v in rows], dtype=np.int32)
    rowptr = np.zeros(n + 1, dtype=np.int64)
    rowptr[1:] = np.cumsum(deg)
    return deg, rowptr, np.concatenate(rows), np.concatenate([np.concatenate(v) for v in imgs])


def cuthill_mckee(rowptr, cols, degree, seed_order=None, reverse=True):
    """Sequential k-d-tree Cuthill-McKee, restating
    InchingLiteInteger/Fuel/Coordinate/T1.py:254-323 over an adjacency list.

    * seeds: next unvisited atom in ``np.argsort(degree)`` order (T1.py:254,261-266);
    * each frontier atom appends its unvisited neighbours in DESCENDING index
      order (query_ball_point(..., return_sorted=True)[::-1], T1.py:276-286);
    * the appended run is insertion-sorted by degree with strict '<' (stable,
      T1.py:289-304);
    * the result is reversed and its inverse permutation returned (T1.py:314-323).
    """
    n = len(degree)
    degree = np.asarray(degree)
    inds = np.argsort(degree) if seed_order is None else np.asarray(seed_order).copy()
    visited = np.zeros(n, dtype=bool)
    order = np.zeros(n, dtype=np.int64)
    N = 0
    for zz in range(n):
        seed = inds[zz]
        if visited[seed]:
            continue
        order[N] = seed
        N += 1
        visited[seed] = True
        ls, le = N - 1, N
        while ls < le:
            for ii in range(ls, le):
                i = order[ii]
                n_old = N
                nb = cols[rowptr[i]:rowptr[i + 1]][::-1]
                for j in nb:
                    if not visited[j]:
                        visited[j] = True
                        order[N] = j
                        N += 1
                seg = order[n_old:N].copy()
                degs = degree[seg]
                # insertion sort, strict '<' == stable sort by degree
                perm = np.argsort(degs, kind="stable")
                order[n_old:N] = seg[perm]
            ls, le = le, N
        if N == n:
            break
    if reverse:
        order = order[::-1].copy()
    return order, np.argsort(order)


def batch_heads(n_atoms: int, maxleafsize: int = 100) -> np.ndarray:
    """Row-batch heads: leaves of the recursive halving tree of
    InchingLiteInteger/util.py:563-571 (left k+1, right n-k-1, k=floor(n/2),
    until <= maxleafsize), sorted descending and cumulated (Fuel/T1.py:145-158)."""
    leaves = []

    def rec(n):
        if n <= maxleafsize:
            leaves.append(n)
            return
        k = n // 2
        rec(k + 1)
        rec(n - k - 1)

    rec(n_atoms)
    heads = [0]
    for s in sorted(leaves)[::-1]:
        heads.append(heads[-1] + s)
    return np.asarray(heads, dtype=np.int64)


def band_slices(rowptr, cols, n_atoms, maxleafsize=100, gap=100):
    """Ungapped per-batch column slices and HalfNnz, restating
    InchingLiteInteger/Fuel/Coordinate/T1.py:371-481 over an adjacency list.
    Returns (dict{batch: [(start, end), ...]}, HalfNnz float)."""
    heads = batch_heads(n_atoms, maxleafsize)
    out = {}
    total = 0
    for b in range(len(heads) - 1):
        start, end = int(heads[b]), int(heads[b + 1])
        flat = cols[rowptr[start]:rowptr[end]]
        total += len(flat)
        uniq = np.unique(flat)
        lo, hi = int(flat.min()), int(flat.max())
        bounds = [lo]
        diffs = np.diff(uniq)
        for iii, xxx in enumerate(diffs):
            if iii == len(uniq) - 5:
                continue
            if iii < 5:
                continue
            if xxx > gap:
                if (bounds[-1] + 5 >= start) and (int(uniq[iii]) + 1 <= start + (end - start) + 5):
                    continue
                bounds.extend([int(uniq[iii]) + 1, int(uniq[iii + 1])])
        bounds.append(hi + 1)
        out[b] = [(bounds[t], bounds[t + 1]) for t in range(0, len(bounds), 2)]
    halfnnz = (((total - n_atoms) / 2) + n_atoms) * 9
    return out, halfnnz


# ---------------------------------------------------------------------------
# C restatement of neighbor_lists / cuthill_mckee (oracle/graph_c.c) for inputs
# of millions of atoms; compiled with gcc on first use into oracle/_build/.
# ---------------------------------------------------------------------------
_CLIB = None


def _clib():
    global _CLIB
    if _CLIB is not None:
        return _CLIB
    import ctypes
    import os
    import subprocess
    here = os.path.dirname(os.path.abspath(__file__))
    src = os.path.join(here, "graph_c.c")
    out_dir = os.path.join(here, "_build")
    so = os.path.join(out_dir, "liboracle_graph.so")
    if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        os.makedirs(out_dir, exist_ok=True)
        tmp = so + f".{os.getpid()}.tmp"
        subprocess.run(["gcc", "-O2", "-shared", "-fPIC", "-o", tmp, src, "-lm"], check=True)
        os.replace(tmp, so)
    L = ctypes.CDLL(so)
    P = ctypes.c_void_p
    L.oracle_neighbor_count.restype = ctypes.c_int64
    L.oracle_neighbor_count.argtypes = [P, ctypes.c_int64, ctypes.c_double, P, P]
    L.oracle_neighbor_fill.restype = ctypes.c_int
    L.oracle_neighbor_fill.argtypes = [P, ctypes.c_int64, ctypes.c_double, P, P]
    L.oracle_cuthill_mckee.restype = ctypes.c_int
    L.oracle_cuthill_mckee.argtypes = [ctypes.c_int64, P, P, P, P, P]
    _CLIB = L
    return L


def neighbor_lists_c(X_nm: np.ndarray, rc_gamma_A: float = 8.0):
    """neighbor_lists() in C: (degree int32, rowptr int64, cols int32)."""
    L = _clib()
    X = np.ascontiguousarray(X_nm, dtype=np.float64)
    n = X.shape[0]
    rc = rc_gamma_A / 10.0
    deg = np.zeros(n, np.int32)
    rowptr = np.zeros(n + 1, np.int64)
    nnz = L.oracle_neighbor_count(X.ctypes.data, n, rc, deg.ctypes.data, rowptr.ctypes.data)
    assert nnz >= 0, "oracle_neighbor_count failed"
    cols = np.zeros(max(nnz, 1), np.int32)[:nnz]
    assert L.oracle_neighbor_fill(X.ctypes.data, n, rc, rowptr.ctypes.data, cols.ctypes.data) == 0
    return deg, rowptr, cols


def cuthill_mckee_c(rowptr, cols, degree, seed_order=None):
    """cuthill_mckee(..., reverse=True) in C: (order int64, undo int64)."""
    L = _clib()
    rowptr = np.ascontiguousarray(rowptr, dtype=np.int64)
    cols = np.ascontiguousarray(cols, dtype=np.int32)
    degree = np.ascontiguousarray(degree, dtype=np.int32)
    n = degree.shape[0]
    seeds = np.ascontiguousarray(np.argsort(degree) if seed_order is None else seed_order, dtype=np.int64)
    order = np.zeros(n, np.int64)
    rc = L.oracle_cuthill_mckee(n, rowptr.ctypes.data, cols.ctypes.data, degree.ctypes.data, seeds.ctypes.data,
                                order.ctypes.data)
    assert rc == 0, f"oracle_cuthill_mckee failed ({rc})"
    return order, np.argsort(order)
