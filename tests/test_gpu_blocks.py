"""Solver building blocks through the C ABI (inch_cheb_filter, inch_cheb_filter_scaled,
inch_block_orth, inch_rr_project / inch_rr_rotate, inch_residual_fp64) against the
same steps done with the package's torch code.  Tolerances: FP64 1e-11 relative,
FP32 filters 1e-4 relative (to the block's norm), orthonormality 1e-12."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small():
    from inching_b200 import graph, synth
    from inching_b200.deflation import rigid_body_basis
    from inching_b200.hessian import HessianStore
    X = synth.globule(1500, seed=19) / 10.0
    order, _ = graph.cuthill_mckee(X, 8.0)
    Xr = torch.from_numpy(X[order.cpu().numpy()]).cuda()
    H = HessianStore(Xr, 8.0, 1.0)
    return dict(H=H, Q=rigid_body_basis(Xr))


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max())


@pytest.mark.parametrize("prec", [64, 32])
def test_cheb_filter_matches_recurrence(small, prec):
    from inching_b200 import _native
    H = small["H"]
    dt = torch.float64 if prec == 64 else torch.float32
    g = torch.Generator(device="cuda").manual_seed(1)
    X = torch.randn(H.shape[0], 72, generator=g, dtype=torch.float64, device="cuda")   # > 64 columns: panels
    mu = np.random.default_rng(2).standard_normal(13)
    cc, dd = 30.0, 31.0
    ent, diag = H.store(prec)
    Y = _native.cheb_filter(prec, H.n_atoms, H.rowptr, ent, diag, X.to(dt).contiguous(), mu, cc, dd).double()
    # reference: the three-term recurrence with FP64 products
    x0, x1 = X, (H.matmul(X, prec=64) - cc * X) / dd
    ref = mu[0] * x0 + mu[1] * x1
    for k in range(1, 12):
        x2 = 2.0 * (H.matmul(x1, prec=64) - cc * x1) / dd - x0
        ref = ref + mu[k + 1] * x2
        x0, x1 = x1, x2
    assert _rel(Y, ref) < (1e-11 if prec == 64 else 1e-4)


@pytest.mark.parametrize("prec", [64, 32])
def test_cheb_filter_scaled_matches_block_solver_filter(small, prec):
    from inching_b200 import _native
    from inching_b200.solvers.chfsi import _Filter
    H = small["H"]
    dt = torch.float64 if prec == 64 else torch.float32
    X = torch.randn(H.shape[0], 40, dtype=torch.float64, device="cuda")
    a, b_up, a0 = 4.0, 62.0, 1.0
    ref = _Filter(H, prec)(X, 9, a, b_up, a0)
    ent, diag = H.store(prec)
    Y = _native.cheb_filter_scaled(prec, H.n_atoms, H.rowptr, ent, diag, X.to(dt).contiguous(), 9, a, b_up,
                                   a0).double()
    assert _rel(Y, ref) < (1e-12 if prec == 64 else 1e-5)


def test_block_orth_deflates_and_orthonormalises(small):
    from inching_b200 import _native
    H, Q = small["H"], small["Q"]
    n = H.shape[0]
    g = torch.Generator(device="cuda").manual_seed(3)
    L, _ = torch.linalg.qr(torch.randn(n, 10, generator=g, dtype=torch.float64, device="cuda"))
    L = L - Q.t() @ (Q @ L)
    L, _ = torch.linalg.qr(L)
    locked = L.t().contiguous()
    # an ill-conditioned block: columns scaled over 7 decades, plus parts in span(Q, locked)
    Y = torch.randn(n, 48, generator=g, dtype=torch.float64, device="cuda") * torch.logspace(0, -7, 48,
                                                                                             dtype=torch.float64,
                                                                                             device="cuda")
    Y = Y + Q.t() @ torch.randn(6, 48, dtype=torch.float64, device="cuda") + L @ torch.randn(10, 48,
                                                                                           dtype=torch.float64,
                                                                                           device="cuda")
    ref = Y - Q.t() @ (Q @ Y)
    ref = ref - L @ (L.t() @ ref)
    ref, _ = torch.linalg.qr(ref)
    Z = _native.block_orth(Y.clone(), B1=Q, B2=locked, passes=3)
    I = torch.eye(48, dtype=torch.float64, device="cuda")
    assert float((Z.t() @ Z - I).abs().max()) < 1e-12
    assert float((Q @ Z).abs().max()) < 1e-12 and float((locked @ Z).abs().max()) < 1e-12
    s = torch.linalg.svdvals(ref.t() @ Z)           # same subspace: all cosines 1
    assert float((1.0 - s).abs().max()) < 1e-9


def test_rr_project_rotate_and_residuals(small):
    from inching_b200 import _native
    H = small["H"]
    Y, _ = torch.linalg.qr(torch.randn(H.shape[0], 30, dtype=torch.float64, device="cuda"))
    Y = Y.contiguous()
    HY = H.matmul(Y, prec=64)
    G = _native.rr_project(Y, HY)
    Gr = Y.t() @ HY
    Gr = 0.5 * (Gr + Gr.t())
    assert _rel(G, Gr) < 1e-13
    th, W = torch.linalg.eigh(Gr)
    Z = _native.rr_rotate(Y, W, 20)
    assert _rel(Z, Y @ W[:, :20]) < 1e-13
    HZ = HY @ W[:, :20]
    res = _native.residual_fp64(HZ.contiguous(), Z, th[:20].contiguous())
    ref = torch.linalg.vector_norm(HZ - Z * th[:20][None, :], dim=0)
    assert _rel(res, ref) < 1e-12
