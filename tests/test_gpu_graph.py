"""GPU parity of the integer/graph path against the reference's golden outputs and
the oracle: neighbour lists, degrees, Cuthill-McKee order, band slices.
Bit-exact comparisons throughout."""
import glob
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from oracle import graph as og

pytestmark = pytest.mark.gpu

FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "rcm_*.npz")))


def _native():
    from inching_b200 import _native
    return _native


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[4:-4])
def test_neighbors_and_rcm_match_reference(path):
    from inching_b200 import graph
    d = np.load(path)
    X = d["X"]
    deg, rowptr, cols = graph.neighbor_lists(X, 8.0)
    assert np.array_equal(deg.cpu().numpy(), d["degree"])
    if "cols" in d:
        assert np.array_equal(rowptr.cpu().numpy(), d["rowptr"])
        assert np.array_equal(cols.cpu().numpy(), d["cols"])
    seeds = torch.from_numpy(d["seed_order"].astype(np.int64)).cuda()
    order, undo, levels = _native().cuthill_mckee(rowptr, cols, deg, seeds)
    assert np.array_equal(order.cpu().numpy(), d["order"])
    assert np.array_equal(undo.cpu().numpy(), d["undo"])
    assert levels >= 1


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p)[4:-4])
def test_band_slices_match_reference(path):
    from inching_b200 import graph
    d = np.load(path)
    X = d["X"]
    Xr = X[d["order"]]
    sl, halfnnz = graph.band_slices(Xr, 8.0, maxleafsize=100, gap=100)
    cnt = np.array([len(sl[i]) for i in range(len(sl))])
    st = np.array([s for i in range(len(sl)) for s, e in sl[i]])
    en = np.array([e for i in range(len(sl)) for s, e in sl[i]])
    assert np.array_equal(cnt, d["slice_counts"])
    assert np.array_equal(st, d["slice_starts"])
    assert np.array_equal(en, d["slice_ends"])
    assert halfnnz == float(d["halfnnz"])
    if "raw_slice_counts" in d:
        sl0, _ = graph.band_slices(X, 8.0, maxleafsize=100, gap=100)
        cnt = np.array([len(sl0[i]) for i in range(len(sl0))])
        st = np.array([s for i in range(len(sl0)) for s, e in sl0[i]])
        assert np.array_equal(cnt, d["raw_slice_counts"])
        assert np.array_equal(st, d["raw_slice_starts"])


def test_reference_facade_cuthill_order_dtypes():
    from inching_b200.Fuel.Coordinate.T1 import X_KdCuthillMckeeOrder
    d = np.load(os.path.join(GOLDEN, "rcm_two_components.npz"))
    order, undo = X_KdCuthillMckeeOrder(d["X"], rc_Gamma=8.0, Reverse=True)
    assert order.dtype == np.int32 and undo.dtype == np.int64
    # the facade seeds with this host's np.argsort, exactly as the reference does
    deg = d["degree"]
    o_ref, u_ref = og.cuthill_mckee(d["rowptr"], d["cols"], deg, seed_order=np.argsort(deg))
    assert np.array_equal(order, o_ref) and np.array_equal(undo, u_ref)
    o2, u2, mean, std = X_KdCuthillMckeeOrder(d["X"], rc_Gamma=8.0, Reverse=False, ReturnStat=True)
    assert np.array_equal(o2, o_ref[::-1]) and abs(mean - deg.mean()) < 1e-12 and abs(std - deg.std()) < 1e-12


def test_neighbors_full_size_assembly100k():
    """Configuration size (100,000 atoms, 20 touching globules): adjacency equals
    scipy cKDTree (the reference's neighbour engine), RCM equals the oracle."""
    from scipy.spatial import cKDTree
    from inching_b200 import graph, synth
    X = synth.workload("assembly100k") / 10.0
    deg, rowptr, cols = graph.neighbor_lists(X, 8.0)
    tree = cKDTree(X)
    nl = tree.query_ball_point(X, 0.8, p=2.0, eps=0, return_sorted=True)
    ref_deg = np.array([len(v) for v in nl], dtype=np.int32)
    assert np.array_equal(deg.cpu().numpy(), ref_deg)
    assert np.array_equal(cols.cpu().numpy(), np.concatenate(nl).astype(np.int32))
    rp, cc = rowptr.cpu().numpy(), cols.cpu().numpy()
    seeds = np.argsort(ref_deg)
    order, undo, levels = _native().cuthill_mckee(rowptr, cols, deg, torch.from_numpy(seeds).cuda())
    o_ref, u_ref = og.cuthill_mckee(rp, cc, ref_deg, seed_order=seeds)
    assert np.array_equal(order.cpu().numpy(), o_ref)
    assert np.array_equal(undo.cpu().numpy(), u_ref)
    # banding property: bandwidth after RCM far below the original
    inv = u_ref
    rows = np.repeat(np.arange(len(ref_deg)), np.diff(rp))
    bw_after = np.abs(inv[rows] - inv[cc]).max()
    assert bw_after < 0.2 * len(ref_deg)


def test_limits_and_bad_input_raise():
    from inching_b200 import graph
    X = np.zeros((4, 3))
    X[1, 0] = np.nan
    with pytest.raises(AssertionError, match="ABORTED"):
        graph.neighbor_lists(X, 8.0)
    # seed order that is not a permutation
    Xg = np.load(os.path.join(GOLDEN, "rcm_near_cutoff.npz"))["X"]
    deg, rowptr, cols = graph.neighbor_lists(Xg, 8.0)
    bad = torch.zeros(deg.shape[0], dtype=torch.int64, device="cuda")
    with pytest.raises(AssertionError, match="permutation"):
        _native().cuthill_mckee(rowptr, cols, deg, bad)


def test_graph_full_size_cube2400k():
    """The largest configuration (2,400,000 atoms, 300 touching globules in a cube;
    81 Cuthill-McKee levels and a band of ~62k atoms, unlike the 100k assembly):
    degrees equal scipy cKDTree's (the reference's neighbour engine), the lists
    equal the C restatement of the oracle, and the Cuthill-McKee order and its
    inverse equal the oracle's, bit for bit."""
    from scipy.spatial import cKDTree
    from inching_b200 import graph, synth
    X = synth.workload("cube2400k") / 10.0
    deg, rowptr, cols = graph.neighbor_lists(X, 8.0)
    deg_h = deg.cpu().numpy()
    ref_len = cKDTree(X).query_ball_point(X, 0.8, p=2.0, eps=0, return_length=True, workers=-1)
    assert np.array_equal(deg_h, ref_len.astype(np.int32))
    d_c, rp_c, c_c = og.neighbor_lists_c(X, 8.0)
    assert np.array_equal(deg_h, d_c)
    assert np.array_equal(rowptr.cpu().numpy(), rp_c)
    assert np.array_equal(cols.cpu().numpy(), c_c)
    seeds = np.argsort(d_c)
    order, undo, levels = _native().cuthill_mckee(rowptr, cols, deg, torch.from_numpy(seeds).cuda())
    o_ref, u_ref = og.cuthill_mckee_c(rp_c, c_c, d_c, seed_order=seeds)
    assert np.array_equal(order.cpu().numpy(), o_ref)
    assert np.array_equal(undo.cpu().numpy(), u_ref)
