"""Drop-in for InchingLiteInteger.Fuel.Coordinate.T1: k-d-tree Cuthill-McKee order
and ungapped band slices, computed by the CUDA cell-list / level-BFS / segmented
sort kernels.  Same names, arguments, defaults, return types and "ABORTED."
assertions as the reference (Fuel/Coordinate/T1.py:171-481).
"""
from __future__ import annotations

import numpy as np
import torch

from ... import graph


def _check_pbc(User_DictCharmmGuiPbc, rc_Gamma):
    """The reference's box-size asserts (Fuel/Coordinate/T1.py:221-222; box in nm,
    compared with rc_Gamma / 10)."""
    if User_DictCharmmGuiPbc is None:
        return None
    bx, by = graph.pbc_box(User_DictCharmmGuiPbc)
    assert bx > rc_Gamma / 10.0, "ABORTED. The PBC box size X is smaller than rc gamma."
    assert by > rc_Gamma / 10.0, "ABORTED. The PBC box size Y is smaller than rc gamma."
    return bx, by


def X_KdCuthillMckeeOrder(X, rc_Gamma=15.0, Reverse=True, ReturnStat=False, User_maxleafsize=1000,
                          User_DictCharmmGuiPbc=None):
    """Reversed (or plain) Cuthill-McKee order of the rc_Gamma (Angstrom) contact
    graph of X (nm, (n_atoms, 3)) and the inverse permutation.

    Returns (order int32, undo int64[, mean degree, std degree]) as numpy arrays,
    like Fuel/Coordinate/T1.py:314-323.  User_maxleafsize only chunked the
    reference's k-d-tree queries; it does not change the result.  With
    User_DictCharmmGuiPbc the graph has periodic xy images; see
    graph.cuthill_mckee for why that order differs from the reference's."""
    pbc = _check_pbc(User_DictCharmmGuiPbc, rc_Gamma)
    order, undo, (degree, _, _, _) = graph.cuthill_mckee(X, rc_Gamma, return_graph=True, pbc=pbc)
    order = order.cpu().numpy()
    if Reverse:
        o = order.astype(np.int32)
        u = undo.cpu().numpy()
    else:
        o = order[::-1].astype(np.int32)
        u = np.argsort(o).astype(np.int64)
    if ReturnStat:
        deg = degree.cpu().numpy()
        return o, u, np.mean(deg), np.std(deg)
    return o, u


def X_KdUngappedMinMaxNeighbor(X, rc_Gamma=15.0, maxleafsize=1000, CollectStat=False, User_ReturnHalfNnz=False,
                               User_GapSize=100, User_DictCharmmGuiPbc=None, SliceForm=True):
    """Per row batch, the list of (start, end) column slices that cover every
    neighbour column with gaps wider than User_GapSize removed; optionally the
    half-store nonzero count HalfNnz = (((sum deg) - n)/2 + n) * 9
    (Fuel/Coordinate/T1.py:331-481)."""
    pbc = _check_pbc(User_DictCharmmGuiPbc, rc_Gamma)
    slices, halfnnz = graph.band_slices(X, rc_Gamma, maxleafsize=maxleafsize, gap=User_GapSize, pbc=pbc)
    if User_ReturnHalfNnz:
        return slices, halfnnz
    return slices
