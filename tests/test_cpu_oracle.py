"""CPU tests: the oracle against the reference's golden outputs, host-side logic,
and the C-ABI library (loads, exports every symbol the header declares)."""
import glob
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
from oracle import graph as og
from oracle import hessian as oh
from oracle import solvers as osv

FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "rcm_*.npz")))


def _slices_arrays(sl):
    cnt = np.array([len(sl[i]) for i in range(len(sl))])
    st = np.array([s for i in range(len(sl)) for s, e in sl[i]])
    en = np.array([e for i in range(len(sl)) for s, e in sl[i]])
    return cnt, st, en


@pytest.mark.parametrize("path", [p for p in FIXTURES if "5k" not in p], ids=lambda p: os.path.basename(p)[4:-4])
def test_oracle_pinned_to_reference(path):
    """Oracle neighbour lists, RCM, band slices and HalfNnz == reference outputs."""
    d = np.load(path)
    X = d["X"]
    deg, rp, c = og.neighbor_lists(X, 8.0)
    assert np.array_equal(deg, d["degree"])
    assert np.array_equal(rp, d["rowptr"]) and np.array_equal(c, d["cols"])
    o, u = og.cuthill_mckee(rp, c, deg, seed_order=d["seed_order"])
    assert np.array_equal(o, d["order"]) and np.array_equal(u, d["undo"])
    _, rpr, cr = og.neighbor_lists(X[o], 8.0)
    sl, hn = og.band_slices(rpr, cr, len(X))
    cnt, st, en = _slices_arrays(sl)
    assert np.array_equal(cnt, d["slice_counts"]) and np.array_equal(st, d["slice_starts"])
    assert np.array_equal(en, d["slice_ends"]) and hn == float(d["halfnnz"])
    sl0, _ = og.band_slices(rp, c, len(X))
    cnt, st, en = _slices_arrays(sl0)
    assert np.array_equal(cnt, d["raw_slice_counts"]) and np.array_equal(st, d["raw_slice_starts"])
    assert np.array_equal(en, d["raw_slice_ends"])


def test_oracle_rcm_config0_size():
    d = np.load(os.path.join(GOLDEN, "rcm_globule5k.npz"))
    deg, rp, c = og.neighbor_lists(d["X"], 8.0)
    assert np.array_equal(deg, d["degree"])
    o, u = og.cuthill_mckee(rp, c, deg, seed_order=d["seed_order"])
    assert np.array_equal(o, d["order"]) and np.array_equal(u, d["undo"])


def test_batch_heads_match_partition_tree():
    from inching_b200 import graph
    for n in (1, 99, 100, 101, 1000, 4999, 5000, 12345):
        for leaf in (100, 1000, 108):
            assert np.array_equal(graph.batch_heads(n, leaf), og.batch_heads(n, leaf))
    # the reference's own tree for 1000 atoms, leaf 100 (util.py:563-571)
    assert graph.partition_tree(1000, 100) == ((((64, 62), (63, 62)), ((64, 62), (63, 61))),
                                               (((64, 62), (63, 61)), ((63, 62), (63, 61))))


def test_oracle_hessian_known_answers():
    from inching_b200 import synth
    X = synth.globule(400, seed=2) / 10.0
    A, Ad = oh.hessian_lower(X)
    H = oh.full_from_lower(A, Ad).toarray()
    assert np.abs(H - H.T).max() == 0.0
    Q = oh.rigid_body_basis(X)
    assert np.abs(H @ Q.T - Q.T).max() < 1e-13
    assert np.abs(Q @ Q.T - np.eye(6)).max() < 1e-13
    v = np.random.default_rng(0).standard_normal(H.shape[0])
    assert np.allclose(oh.krylov_av(A, Ad, v), H @ v, rtol=0, atol=1e-12)


def test_oracle_solvers_vs_dense_eigh():
    from inching_b200 import synth
    X = synth.globule(300, seed=4) / 10.0
    A, Ad = oh.hessian_lower(X)
    H = oh.full_from_lower(A, Ad).toarray()
    w = np.linalg.eigvalsh(H)
    Q = oh.rigid_body_basis(X)
    op = lambda v: oh.krylov_av(A, Ad, v)
    S, V, _ = osv.trlm(op, H.shape[0], k=8, tol=1e-9, Q=Q, shift=10.0)
    assert np.abs(S - w[6:14]).max() < 1e-10
    S2, V2, _, conv = osv.jdm(op, H.shape[0], k=8, tol=1e-9, Q=Q, shift=10.0)
    assert conv and np.abs(S2 - w[6:14]).max() < 1e-10
    lo, hi = osv.spectrum_bound(op, H.shape[0], steps=100)
    assert abs(hi - w[-1]) < 1e-8 * w[-1] and abs(lo - w[0]) < 1e-6


def _header_symbols():
    syms = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        syms |= set(re.findall(r"\b(inch_[a-z0-9_]+)\s*\(", txt))
    return syms


def test_library_exports_header_symbols():
    import ctypes
    from inching_b200 import _native
    lib = _native.lib()
    syms = _header_symbols()
    assert len(syms) >= 10
    for s in sorted(syms):
        assert hasattr(lib, s), s
    assert set(_native.exported_symbols()) == syms
    assert lib.inch_abi_version() >= 1
    assert isinstance(lib.inch_last_error_string(), bytes)
    # size queries need no GPU
    assert _native.lib().inch_rcm_workspace_size(1000) > 4 * 1000 * 3


def test_no_cuda_means_loud_failure():
    import torch
    if torch.cuda.is_available():
        pytest.skip("only meaningful without a GPU")
    from inching_b200 import graph
    with pytest.raises(RuntimeError, match="CUDA"):
        graph.neighbor_lists(np.zeros((3, 3)), 8.0)


def test_oracle_cdm_matches_dense():
    """The oracle's Chebyshev-Davidson restatement (reference flow, including its
    post-convergence filter input) against LAPACK on a 300-atom globule."""
    from inching_b200 import synth
    from oracle import hessian as oh
    from oracle import solvers as osv
    X = synth.globule(300, seed=2) / 10.0
    A, Ad = oh.hessian_lower(X, 8.0, 1.0)
    H = oh.full_from_lower(A, Ad)
    w = np.linalg.eigvalsh(H.toarray())
    lam, V, its, ok = osv.cdm(lambda v: H @ v, H.shape[0], k=10, tol=1e-10, degree=16,
                              spectrum_bound=(w[0], w[-1]))
    assert ok
    assert np.abs(lam - w[:10]).max() < 1e-9 * w[-1]
    R = H @ V - V * lam[None, :]
    assert np.linalg.norm(R, axis=0).max() < 1e-8 * w[-1]


def test_oracle_pbc_xy_neighbours_match_reference_golden():
    """Periodic xy neighbour lists: the oracle's restatement against the lists the
    reference's X_cKDTreePbcXy produced (degree pass form: per image sorted,
    images concatenated in instruction order)."""
    g = np.load(os.path.join(GOLDEN, "pbc_slab.npz"))
    deg, rowptr, cols, image = og.neighbor_lists_pbc_xy(g["X"], 8.0, g["box"][:2])
    assert np.array_equal(deg, g["degree"])
    assert np.array_equal(cols, g["cols"])
    # some rows really use images, and within a row each image block is sorted
    assert (image > 0).sum() > 0.1 * len(image)
    for i in range(0, len(deg), 97):
        seg_c, seg_i = cols[rowptr[i]:rowptr[i + 1]], image[rowptr[i]:rowptr[i + 1]]
        assert np.all(np.diff(seg_i) >= 0)
        for k in np.unique(seg_i):
            assert np.all(np.diff(seg_c[seg_i == k]) > 0)


def test_oracle_pbc_hessian_translation_invariant():
    """With periodic images the three translations stay null vectors of the ANM
    part (rotations do not): H t = PlusI t."""
    g = np.load(os.path.join(GOLDEN, "pbc_slab.npz"))
    X = g["X"][:600] * np.array([1.0, 1.0, 1.0])
    A, Ad = oh.hessian_lower(X, 8.0, 1.0, box_xy=g["box"][:2])
    H = oh.full_from_lower(A, Ad)
    n = X.shape[0]
    for a in range(3):
        t = np.zeros((n, 3))
        t[:, a] = 1.0
        t = t.ravel()
        assert np.abs(H @ t - t).max() < 1e-10
    r = np.cross(X - X.mean(0), np.array([0.0, 0.0, 1.0])).ravel()
    assert np.abs(H @ r - r).max() > 1e-3
