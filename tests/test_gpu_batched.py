"""Batched many-structure solve (block-diagonal store, one SpMM launch per
Chebyshev step for a whole bucket) against per-structure dense LAPACK eigh.
Tolerances: mixed precision at residual 1e-6*||H|| -> relative eigenvalue error
<= 1e-6; FP64 at 1e-9*||H|| -> 1e-10."""
import numpy as np
import pytest

from oracle import hessian as oh

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,tol,eig_tol", [("f64", 1e-9, 1e-10), ("mixed", 1e-6, 1e-6)])
def test_batched_matches_dense(precision, tol, eig_tol):
    from inching_b200 import synth
    from inching_b200.batched import batched_normal_modes
    sizes = synth.batch_sizes(14, 300, 1200, seed=5)
    structs = [synth.globule(int(n), seed=100 + i) / 10.0 for i, n in enumerate(sizes)]
    res, info = batched_normal_modes(structs, k=12, tol=tol, precision=precision, bucket_ratio=1.6)
    assert len(info["buckets"]) >= 2
    for X, (ev, modes) in zip(structs, res):
        A, Ad = oh.hessian_lower(X, 8.0, 1.0)
        Hd = oh.full_from_lower(A, Ad).toarray()
        w = np.linalg.eigvalsh(Hd)
        ref = w[6:18] - 1.0
        assert np.max(np.abs(ev - ref) / np.abs(ref)) < eig_tol
        V = modes.reshape(12, -1).cpu().numpy()
        Q = oh.rigid_body_basis(X)
        assert np.abs(Q @ V.T).max() < 1e-6
        r = np.linalg.norm(Hd @ V.T - V.T * (ev + 1.0)[None, :], axis=0)
        assert r.max() <= tol * 1.5 * w[-1] * 1.05
