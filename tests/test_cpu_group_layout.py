"""The row-group store format on the CPU: what the device builder writes (group_ptr,
R weight slots per union, slot 0 holding the column, zero slots where a row lacks
the column, each group padded with zero-weight unions to a multiple of 16) is a
lossless rearrangement of the rank-one pair store.

A host restatement of the merge is walked in FP64 and compared with the oracle's
Krylov product (restatement of Krylov/T3.py:128-160) to 1e-12 relative to
||H|| |X|; the merge keeps each row's entries in their adjacency order, the
property the device product relies on for the pair kernel's bits."""
import numpy as np
import pytest

from oracle import graph as og
from oracle import hessian as oh

PAD = 16


def _pair_weights(X, rowptr, cols):
    """w = (x_j - x_i) / |x_j - x_i| per adjacency entry (0 for the self entry)."""
    rows = np.repeat(np.arange(X.shape[0]), np.diff(rowptr))
    d = X[cols] - X[rows]
    r = np.sqrt((d * d).sum(axis=1))
    w = np.zeros_like(d)
    nz = r > 0
    w[nz] = d[nz] / r[nz, None]
    return rows, w


def _merge(rowptr, cols, w, n, R):
    """(group_ptr, union columns, slots (U, R, 3), per-row taken entry order, real
    unions per group before the padding)."""
    gptr, gcol, slots, order, nreal = [0], [], [], {i: [] for i in range(n)}, []
    for g in range((n + R - 1) // R):
        rows = list(range(R * g, min(R * g + R, n)))
        pos = {r: int(rowptr[r]) for r in rows}
        cnt = 0
        while True:
            heads = {r: int(cols[pos[r]]) for r in rows if pos[r] < rowptr[r + 1]}
            if not heads:
                break
            m = min(heads.values())
            s = np.zeros((R, 3))
            for r, h in heads.items():
                if h == m:
                    s[r - R * g] = w[pos[r]]
                    order[r].append(pos[r])
                    pos[r] += 1
            gcol.append(m)
            slots.append(s)
            cnt += 1
        nreal.append(cnt)
        while cnt % PAD:
            gcol.append(R * g)
            slots.append(np.zeros((R, 3)))
            cnt += 1
        gptr.append(gptr[-1] + cnt)
    return np.array(gptr), np.array(gcol), np.array(slots), order, nreal


def _group_product(X, rowptr, cols, w, plus_i, gptr, gcol, slots, V, R):
    n = X.shape[0]
    rows = np.repeat(np.arange(n), np.diff(rowptr))
    D = np.zeros((n, 3, 3))
    np.add.at(D, rows, w[:, :, None] * w[:, None, :])
    D += plus_i * np.eye(3)
    Vb = V.reshape(n, 3, -1)
    Y = np.einsum("iab,ibc->iac", D, Vb)
    for g in range(len(gptr) - 1):
        for u in range(gptr[g], gptr[g + 1]):
            xj = Vb[gcol[u]]
            for r in range(R):
                i = R * g + r
                if i < n:
                    wr = slots[u, r]
                    Y[i] -= np.outer(wr, wr @ xj)
    return Y.reshape(3 * n, -1)


@pytest.mark.parametrize("R", [2, 4])
def test_group_format_is_the_pair_store_rearranged(R):
    rng = np.random.default_rng(R)
    n = 301                                          # a partial last group for R = 2 and 4
    X = rng.random((n, 3)) * 2.2
    X[7] = X[3]                                      # coincident pair: d = 0, no spring
    X[-1] += 6.0                                     # isolated atom
    deg, rowptr, cols = og.neighbor_lists(X, 8.0)
    order, _ = og.cuthill_mckee(rowptr, cols, deg)   # banded rows, as the pipeline orders them
    X = X[order]
    deg, rowptr, cols = og.neighbor_lists(X, 8.0)
    _, w = _pair_weights(X, rowptr, cols)
    gptr, gcol, slots, order, nreal = _merge(rowptr, cols, w, n, R)
    assert (np.diff(gptr) % PAD == 0).all() and gptr[-1] == len(gcol)
    # every row's entries are taken once each, in adjacency order
    for i in range(n):
        assert order[i] == list(range(rowptr[i], rowptr[i + 1]))
    # unions are sorted by column within a group up to the padding, which points at the
    # group's first atom and carries no weight
    for g in range(len(gptr) - 1):
        body = gcol[gptr[g]:gptr[g] + nreal[g]]
        assert (np.diff(body) >= 0).all()
        assert (gcol[gptr[g] + nreal[g]:gptr[g + 1]] == R * g).all()
        assert not slots[gptr[g] + nreal[g]:gptr[g + 1]].any()
    assert sum(nreal) < 0.9 * len(cols)              # banded rows share unions
    A, Ad = oh.hessian_lower(X, 8.0, 1.0)
    V = rng.standard_normal((3 * n, 5))
    ref = np.stack([oh.krylov_av(A, Ad, V[:, c]) for c in range(5)], axis=1)
    Y = _group_product(X, rowptr, cols, w, 1.0, gptr, gcol, slots, V, R)
    scale = float(abs(oh.full_from_lower(A, Ad)).max())
    assert np.abs(Y - ref).max() <= 1e-12 * scale * np.abs(V).max() * 10
