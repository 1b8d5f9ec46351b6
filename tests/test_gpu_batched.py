"""Batched many-structure solve (block-diagonal store, one SpMM launch per
Chebyshev step for a whole bucket) against per-structure dense LAPACK eigh.
Tolerances: mixed precision at residual 1e-6*||H|| -> relative eigenvalue error
<= 1e-6; FP64 at 1e-9*||H|| -> 1e-10."""
import numpy as np
import pytest
import torch

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


@pytest.mark.parametrize("prec", [64, 32])
def test_segmented_epilogue_matches_oracle(prec):
    """inch_spmm_seg: per-structure (alpha, gamma, beta) on a block-diagonal store."""
    import torch
    from inching_b200 import synth
    from inching_b200.batched import lattice_layout
    from inching_b200.hessian import HessianStore
    structs = [synth.globule(n, seed=70 + n) / 10.0 for n in (300, 420, 500)]
    Xc = lattice_layout(structs, 0.8)
    H = HessianStore(Xc, 8.0, 1.0)
    A, Ad = oh.hessian_lower(Xc, 8.0, 1.0)
    sizes = np.array([x.shape[0] for x in structs])
    seg = np.repeat(np.arange(3), sizes).astype(np.int32)
    coef = np.array([[0.5, -1.0, 0.25], [2.0, 0.5, -1.0], [-0.75, 0.1, 0.0]])
    rng = np.random.default_rng(4)
    Xv = rng.standard_normal((H.shape[0], 24))
    Yin = rng.standard_normal((H.shape[0], 24))
    HX = np.stack([oh.krylov_av(A, Ad, Xv[:, c]) for c in range(24)], axis=1)
    d = np.repeat(seg, 3)
    ref = coef[d, 0][:, None] * HX + coef[d, 1][:, None] * Xv + coef[d, 2][:, None] * Yin
    dt = torch.float64 if prec == 64 else torch.float32
    Xt = torch.from_numpy(Xv).to("cuda", dt).contiguous()
    Yt = torch.from_numpy(Yin).to("cuda", dt).contiguous()
    H.matmul_seg(Xt, Yt, torch.from_numpy(seg).cuda(), torch.from_numpy(coef).cuda(), Yin=Yt, prec=prec)
    tol = (1e-12 if prec == 64 else 2e-6) * np.abs(ref).max() * 50
    assert np.abs(Yt.double().cpu().numpy() - ref).max() <= tol


def test_sharded_batch_in_one_process_equals_batched():
    """With one process the sharded entry point takes every structure and its
    gathered host results equal the batched solve's."""
    from inching_b200 import synth
    from inching_b200.batched import batched_normal_modes, sharded_batched_normal_modes
    structs = [synth.globule(n, seed=70 + i) / 10.0 for i, n in enumerate([400, 900, 650, 1500])]
    res, _ = batched_normal_modes(structs, k=8, tol=1e-8, precision="f64")
    merged, info = sharded_batched_normal_modes(structs, k=8, tol=1e-8, precision="f64")
    assert info["indices"] == [0, 1, 2, 3] and sorted(merged) == [0, 1, 2, 3]
    for i, (ev, modes) in enumerate(res):
        ev2, m2 = merged[i]
        assert np.max(np.abs(ev2 - ev) / ev) < 1e-9
        assert m2.shape == tuple(modes.shape)


@pytest.mark.parametrize("p", [1, 2, 37, 48, 64])
def test_jacobi_batched_small_eigh(p):
    """The batched Jacobi kernel against LAPACK on random symmetric matrices and on
    ones with a repeated eigenvalue: eigenvalues to 1e-12 of the norm, orthonormal
    eigenvectors, residual A V - V W to 1e-12 of the norm."""
    from inching_b200 import _native
    rng = np.random.default_rng(p)
    A = rng.standard_normal((40, p, p))
    A = A + A.transpose(0, 2, 1)
    Q, _ = np.linalg.qr(rng.standard_normal((p, p)))
    d = np.arange(p, dtype=float) // 2           # pairs of equal eigenvalues
    A[0] = (Q * d) @ Q.T
    G = torch.from_numpy(A).cuda()
    W, V, sw = _native.eigh_batched_small(G, return_sweeps=True)
    W, V = W.cpu().numpy(), V.cpu().numpy()
    w_ref = np.linalg.eigvalsh(A)
    nrm = np.abs(A).max()
    assert np.abs(W - w_ref).max() < 1e-12 * nrm * p
    I = np.eye(p)
    assert np.abs(np.einsum("sji,sjk->sik", V, V) - I).max() < 1e-12 * p
    R = np.einsum("sij,sjk->sik", A, V) - V * W[:, None, :]
    assert np.abs(R).max() < 1e-12 * nrm * p
    assert int(sw.max()) <= 30
