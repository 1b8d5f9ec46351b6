"""Neighbour search, Cuthill-McKee banding, row-batch heads and band slices.

Device work runs in libinching_b200 (cell-list neighbour search, level-synchronous
Cuthill-McKee, segmented-sort band slices).  The host keeps only what the
reference computes with numpy on the host as well: ``np.argsort(degree)`` (its
unstable tie order picks the BFS seeds, InchingLiteInteger/Fuel/Coordinate/T1.py:254)
and the recursive partition tree of the row batches (util.py:563-589).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _native


def _device(device=None):
    if device is None:
        if not torch.cuda.is_available():
            raise RuntimeError("inching_b200 needs a CUDA device (there is no CPU path)")
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device(device)


def to_device_coords(X, device=None) -> torch.Tensor:
    """(N,3) float64 nm coordinates as a contiguous CUDA tensor."""
    dev = _device(device)
    if isinstance(X, torch.Tensor):
        t = X.detach().to(device=dev, dtype=torch.float64)
    else:
        t = torch.from_numpy(np.ascontiguousarray(np.asarray(X, dtype=np.float64))).to(dev)
    t = t.contiguous()
    if t.dim() != 2 or t.shape[1] != 3:
        raise AssertionError("ABORTED. X must have shape (n_atoms, 3)")
    if t.shape[0] < 1:
        raise AssertionError("ABORTED. X has no atoms")
    return t


def pbc_box(pbc):
    """(box_x, box_y) in nm from the reference's User_DictCharmmGuiPbc
    (RectBox_Xsize / RectBox_Ysize, same unit as X) or a (box_x, box_y) pair;
    None stays None."""
    if pbc is None:
        return None
    if isinstance(pbc, dict):
        return float(pbc["RectBox_Xsize"]), float(pbc["RectBox_Ysize"])
    return float(pbc[0]), float(pbc[1])


def neighbor_lists(X, rc_gamma_A: float = 8.0, device=None, pbc=None):
    """Sorted neighbour lists within rc_Gamma (Angstrom; coordinates in nm), self
    included.  Returns device tensors (degree int32, rowptr int64, cols int32);
    with pbc (User_DictCharmmGuiPbc or (box_x, box_y)) the periodic xy images
    too, each row listing image 0's neighbours then image 1's, ..., and a fourth
    tensor with every entry's image code (int8)."""
    Xd = to_device_coords(X, device)
    return _native.neighbor_lists(Xd, rc_gamma_A / 10.0, box_xy=pbc_box(pbc))


def seed_order(degree: torch.Tensor) -> np.ndarray:
    """np.argsort(degree), exactly the reference's call (default kind)."""
    return np.argsort(degree.cpu().numpy())


def cuthill_mckee(X, rc_gamma_A: float = 8.0, device=None, return_graph=False, pbc=None):
    """Reversed Cuthill-McKee order of the cutoff graph of X (nm) and its inverse,
    both as device int64 tensors (plus degree/rowptr/cols when return_graph).

    With pbc the graph includes the periodic xy images.  The order is then a
    valid reversed Cuthill-McKee order of that graph but not the reference's:
    under PBC the reference's BFS reads each parent's neighbours in k-d-tree
    traversal order (single-point queries there ignore return_sorted,
    Fuel/Coordinate/T1.py:130-146), which this level-synchronous BFS does not
    reproduce; degrees and neighbour sets are the reference's exactly."""
    degree, rowptr, cols = neighbor_lists(X, rc_gamma_A, device, pbc=pbc)[:3]
    seeds = torch.from_numpy(seed_order(degree).astype(np.int64)).to(degree.device)
    order, undo, levels = _native.cuthill_mckee(rowptr, cols, degree, seeds)
    if return_graph:
        return order, undo, (degree, rowptr, cols, levels)
    return order, undo


def partition_tree(n: int, maxleafsize: int = 108):
    """Nested tuple of leaf sizes: recursive halving, left k+1 and right n-k-1 with
    k = floor(n/2), until a part has at most maxleafsize rows (util.py:563-571)."""
    if n <= maxleafsize:
        return n
    k = n // 2
    return partition_tree(k + 1, maxleafsize), partition_tree(n - k - 1, maxleafsize)


def flatten_partition_tree(nested):
    """Leaves of a partition tree in left-to-right order (util.py:574-589)."""
    if isinstance(nested, tuple):
        for x in nested:
            yield from flatten_partition_tree(x)
    else:
        yield nested


def batch_heads(n_atoms: int, maxleafsize: int = 100) -> np.ndarray:
    """Row-batch heads: leaf sizes sorted descending, cumulated (Fuel/T1.py:145-158)."""
    heads = [0]
    for s in sorted(flatten_partition_tree(partition_tree(n_atoms, maxleafsize)))[::-1]:
        heads.append(heads[-1] + s)
    return np.asarray(heads, dtype=np.int64)


def band_slices(X, rc_gamma_A: float = 8.0, maxleafsize: int = 1000, gap: int = 100, device=None,
                graph=None, pbc=None):
    """Ungapped column slices per row batch and HalfNnz, as
    X_KdUngappedMinMaxNeighbor (Fuel/Coordinate/T1.py:331-481) returns them
    (with pbc, over the neighbour lists that include periodic xy images)."""
    if graph is None:
        degree, rowptr, cols = neighbor_lists(X, rc_gamma_A, device, pbc=pbc)[:3]
    else:
        degree, rowptr, cols = graph[:3]
    n = degree.shape[0]
    heads = torch.from_numpy(batch_heads(n, maxleafsize)).to(rowptr.device)
    max_slices = 256
    counts, starts, ends, total = _native.band_slices(rowptr, cols, n, heads, gap, max_slices)
    counts = counts.cpu().numpy()
    starts = starts.cpu().numpy()
    ends = ends.cpu().numpy()
    out = {}
    for b in range(len(counts)):
        out[b] = [(int(starts[b, t]), int(ends[b, t])) for t in range(counts[b])]
    halfnnz = (((total - n) / 2) + n) * 9
    return out, halfnnz
