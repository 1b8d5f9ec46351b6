"""Periodic xy images (membrane systems): neighbour lists bit-exact against the
lists the reference's X_cKDTreePbcXy produced, the Hessian against the oracle's
restatement of the reference's image loop, translation invariance, a valid
banding order, and normal modes against dense LAPACK.  Tolerances: integer data
exact; Hessian products 1e-12 relative; eigenvalues 1e-9 relative."""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from oracle import graph as og
from oracle import hessian as oh

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def slab():
    g = np.load(os.path.join(GOLDEN, "pbc_slab.npz"))
    box = g["box"]
    d = {"RectBox_Xsize": box[0], "RectBox_Ysize": box[1], "RectBox_Zsize": box[2],
         "X": (0.0, box[0]), "Y": (0.0, box[1]), "Z": (0.0, box[2])}
    return dict(X=g["X"], box=box, dict=d, degree=g["degree"], cols=g["cols"])


def test_pbc_neighbours_match_reference(slab):
    from inching_b200 import graph
    deg, rowptr, cols, image = graph.neighbor_lists(slab["X"], 8.0, pbc=slab["dict"])
    assert np.array_equal(deg.cpu().numpy(), slab["degree"])
    assert np.array_equal(cols.cpu().numpy(), slab["cols"])
    _, rp_o, _, im_o = og.neighbor_lists_pbc_xy(slab["X"], 8.0, slab["box"][:2])
    assert np.array_equal(rowptr.cpu().numpy(), rp_o)
    assert np.array_equal(image.cpu().numpy(), im_o)


def test_pbc_box_smaller_than_cutoff_is_refused(slab):
    from inching_b200 import graph
    with pytest.raises(AssertionError, match="ABORTED. The PBC box size X"):
        graph.neighbor_lists(slab["X"], 8.0, pbc=(0.79, 3.0))
    from inching_b200.Fuel.Coordinate.T1 import X_KdCuthillMckeeOrder
    with pytest.raises(AssertionError, match="ABORTED. The PBC box size Y"):
        X_KdCuthillMckeeOrder(slab["X"], rc_Gamma=8.0, User_DictCharmmGuiPbc=dict(slab["dict"], RectBox_Ysize=0.5))


def test_pbc_hessian_matches_oracle_and_is_translation_invariant(slab):
    from inching_b200.hessian import HessianStore
    X = slab["X"]
    H = HessianStore(X, 8.0, 1.0, pbc=slab["dict"])
    A, Ad = oh.hessian_lower(X, 8.0, 1.0, box_xy=slab["box"][:2])
    Hs = oh.full_from_lower(A, Ad)
    V = np.random.default_rng(1).standard_normal((Hs.shape[0], 4))
    Y = H.matmul(torch.from_numpy(V).cuda().contiguous(), prec=64).cpu().numpy()
    ref = Hs @ V
    assert np.abs(Y - ref).max() <= 1e-12 * np.abs(ref).max()
    Y32 = H.matmul(torch.from_numpy(V).float().cuda().contiguous(), prec=32).double().cpu().numpy()
    assert np.abs(Y32 - ref).max() <= 1e-5 * np.abs(ref).max()
    n = X.shape[0]
    T = np.zeros((3 * n, 3))
    for a in range(3):
        T[a::3, a] = 1.0
    HT = H.matmul(torch.from_numpy(T).cuda().contiguous(), prec=64).cpu().numpy()
    assert np.abs(HT - T).max() < 1e-10


def test_pbc_ordering_is_a_banding_permutation(slab):
    from inching_b200 import graph
    X = slab["X"]
    order, undo = graph.cuthill_mckee(X, 8.0, pbc=slab["dict"])
    o = order.cpu().numpy()
    assert np.array_equal(np.sort(o), np.arange(len(o)))
    assert np.array_equal(undo.cpu().numpy()[o], np.arange(len(o)))
    deg, rowptr, cols, _ = og.neighbor_lists_pbc_xy(X, 8.0, slab["box"][:2])
    rows = np.repeat(np.arange(len(deg)), np.diff(rowptr))
    bw0 = np.abs(rows - cols).max()
    u = undo.cpu().numpy()
    bw1 = np.abs(u[rows] - u[cols]).max()
    assert bw1 < 0.6 * bw0


def test_pbc_normal_modes_match_dense(slab):
    """Lowest non-translational modes of a 600-atom periodic slab: only the three
    translations are null (rotations are broken by the image bonds)."""
    from inching_b200.pipeline import normal_modes_device
    X = np.ascontiguousarray(slab["X"][:600])
    A, Ad = oh.hessian_lower(X, 8.0, 1.0, box_xy=slab["box"][:2])
    w = np.linalg.eigvalsh(oh.full_from_lower(A, Ad).toarray())
    assert np.abs(w[:3] - 1.0).max() < 1e-10 and w[3] > 1.0 + 1e-6
    ev, modes, info = normal_modes_device(torch.from_numpy(X).cuda(), 10, pbc=slab["dict"], precision="f64",
                                          tol=1e-10)
    assert np.max(np.abs(ev.cpu().numpy() + 1.0 - w[3:13]) / w[3:13]) < 1e-9
    M = modes.cpu().numpy().reshape(10, -1)
    assert np.abs(M.reshape(10, -1, 3).sum(axis=1)).max() < 1e-8
