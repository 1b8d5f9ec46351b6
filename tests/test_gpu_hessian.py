"""GPU parity of the Hessian store and the fused SpMM against the FP64 oracle
(restatement of Fuel/T1.py:276-455 and Krylov/T3.py:128-160).

Tolerances: FP64 store/products 1e-12 relative to ||H||; FP32 store/products
2e-6 relative to ||H|| (single-precision rounding of w and of the sums)."""
import numpy as np
import pytest
import torch

from oracle import hessian as oh

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-6


@pytest.fixture(scope="module")
def case():
    from inching_b200 import graph, synth
    from inching_b200.hessian import HessianStore
    X = synth.globule(1500, seed=7) / 10.0
    order, undo = graph.cuthill_mckee(X, 8.0)
    Xr = X[order.cpu().numpy()]
    H = HessianStore(Xr, 8.0, plus_i=1.0)
    A, Ad = oh.hessian_lower(Xr, 8.0, 1.0)
    Hfull = oh.full_from_lower(A, Ad)
    Q = oh.rigid_body_basis(Xr)
    return Xr, H, A, Ad, Hfull, Q


def test_store_matches_oracle(case):
    Xr, H, A, Ad, Hfull, Q = case
    L = H.to_scipy_lower()
    scale = abs(Hfull).max()
    diff = abs(L - A)
    assert diff.max() <= TOL64 * scale
    assert np.allclose(H.A_diag.cpu().numpy(), Ad, rtol=0, atol=TOL64 * scale)


def test_rigid_body_null_space_and_symmetry(case):
    Xr, H, A, Ad, Hfull, Q = case
    Qt = torch.from_numpy(Q.T.copy()).cuda()
    Y = H.matmul(Qt)
    assert torch.allclose(Y, Qt * H.plus_i, atol=1e-12, rtol=0)
    v = torch.randn(H.shape[0], 2, dtype=torch.float64, device="cuda")
    Hv = H.matmul(v.contiguous())
    assert abs(float(v[:, 0] @ Hv[:, 1] - v[:, 1] @ Hv[:, 0])) < 1e-10


@pytest.mark.parametrize("b", [1, 2, 3, 8, 13, 16, 40, 64, 128, 136, 200])
@pytest.mark.parametrize("prec", [64, 32])
def test_spmm_matches_krylov_av(case, b, prec):
    """Every tile width of the pair kernel (FP32 128-column float4 tiles included)
    against the oracle's Krylov operator."""
    Xr, H, A, Ad, Hfull, Q = case
    rng = np.random.default_rng(b)
    Xv = rng.standard_normal((H.shape[0], b))
    ref = np.stack([oh.krylov_av(A, Ad, Xv[:, c]) for c in range(b)], axis=1)
    dt = torch.float64 if prec == 64 else torch.float32
    Xt = torch.from_numpy(Xv).to("cuda", dt)
    if b == 1:
        Xt = Xt[:, 0].contiguous()
        ref = ref[:, 0]
    Y = H.matmul(Xt, prec=prec)
    tol = (TOL64 if prec == 64 else TOL32) * abs(Hfull).max() * np.abs(Xv).max() * 10
    assert np.abs(Y.double().cpu().numpy() - ref).max() <= tol


@pytest.mark.parametrize("b", [4, 128])
@pytest.mark.parametrize("prec", [64, 32])
def test_spmm_fused_epilogue(case, prec, b):
    """Y = a*HX + g*X + b*Yin + s*Q^T Q X and Acc += mu*Y in one call, vs the oracle
    composition (Krylov/T3.py + Orthogonalization/T3.py + PolynomialFilters/T2.py)."""
    Xr, H, A, Ad, Hfull, Q = case
    rng = np.random.default_rng(3)
    Xv = rng.standard_normal((H.shape[0], b))
    Yin = rng.standard_normal((H.shape[0], b))
    Acc0 = rng.standard_normal((H.shape[0], b))
    a, g, be, s, mu = 0.37, -1.25, -1.0, 10.0, 0.6
    HX = np.stack([oh.krylov_av(A, Ad, Xv[:, c]) for c in range(b)], axis=1)
    ref = a * HX + g * Xv + be * Yin + s * Q.T @ (Q @ Xv)
    dt = torch.float64 if prec == 64 else torch.float32
    t = lambda m: torch.from_numpy(m).to("cuda", dt).contiguous()
    Xt, Yt, Acc = t(Xv), t(Yin), t(Acc0)
    Qd = torch.from_numpy(Q).cuda()
    H.matmul(Xt, out=Yt, prec=prec, alpha=a, gamma=g, beta=be, Yin=Yt, acc=Acc, mu=mu, Q=Qd, hot_shift=s)
    tol = (TOL64 if prec == 64 else TOL32) * abs(Hfull).max() * 50
    assert np.abs(Yt.double().cpu().numpy() - ref).max() <= tol
    assert np.abs(Acc.double().cpu().numpy() - (Acc0 + mu * ref)).max() <= tol


def test_full_size_store_properties():
    """100,000-atom assembly: symmetry via random bilinear forms and the six
    rigid-body vectors as exact eigenvectors (H q = PlusI q), FP64 and FP32."""
    from inching_b200 import graph, synth
    from inching_b200.hessian import HessianStore
    X = synth.workload("assembly100k") / 10.0
    order, _ = graph.cuthill_mckee(X, 8.0)
    Xr = X[order.cpu().numpy()]
    H = HessianStore(Xr, 8.0, plus_i=1.0)
    Q = torch.from_numpy(oh.rigid_body_basis(Xr).T.copy()).cuda()
    Y = H.matmul(Q)
    assert (Y - Q).abs().max().item() < 1e-11
    Y32 = H.matmul(Q.float().contiguous(), prec=32)
    assert (Y32.double() - Q).abs().max().item() < 1e-4
    v = torch.randn(H.shape[0], 2, dtype=torch.float64, device="cuda").contiguous()
    Hv = H.matmul(v)
    assert abs(float(v[:, 0] @ Hv[:, 1] - v[:, 1] @ Hv[:, 0])) < 1e-8 * float(v[:, 0] @ Hv[:, 0])


@pytest.mark.parametrize("prec", [64, 32])
def test_spmm_unaligned_rows_scalar_gather(case, prec):
    """Odd leading dimension (rows not 2-element aligned): the column kernel falls
    back to scalar gathers and must give the same product."""
    from inching_b200 import _native
    Xr, H, A, Ad, Hfull, Q = case
    b, ld = 24, 25
    rng = np.random.default_rng(11)
    Xv = rng.standard_normal((H.shape[0], ld))
    ref = np.stack([oh.krylov_av(A, Ad, Xv[:, c]) for c in range(b)], axis=1)
    dt = torch.float64 if prec == 64 else torch.float32
    Xt = torch.from_numpy(Xv).to("cuda", dt)
    Yt = torch.zeros_like(Xt)
    ent, diag = H.store(prec)
    _native.spmm(prec, H.n_atoms, H.rowptr, ent, diag, Xt[:, :b], Yt[:, :b])
    tol = (TOL64 if prec == 64 else TOL32) * abs(Hfull).max() * np.abs(Xv).max() * 10
    assert np.abs(Yt[:, :b].double().cpu().numpy() - ref).max() <= tol
    assert float(Yt[:, b:].abs().max()) == 0.0


@pytest.mark.parametrize("prec", [64, 32])
@pytest.mark.parametrize("b", [8, 40, 64])
def test_row_tile_layout_matches_oracle(case, prec, b):
    """The optional row-tile layout (8-row tiles, merged neighbour unions) gives the
    same products as the oracle, with the fused epilogue."""
    from inching_b200.hessian import HessianStore
    Xr, H, A, Ad, Hfull, Q = case
    Ht = HessianStore(Xr, 8.0, plus_i=1.0, tiles=True)
    assert Ht.tiles["n_pairs"] == Ht.nnz_blocks - Ht.n_atoms
    rng = np.random.default_rng(b)
    Xv = rng.standard_normal((H.shape[0], b))
    Yin = rng.standard_normal((H.shape[0], b))
    HX = np.stack([oh.krylov_av(A, Ad, Xv[:, c]) for c in range(b)], axis=1)
    ref = 0.5 * HX - 0.25 * Xv - Yin + 10.0 * Q.T @ (Q @ Xv)
    dt = torch.float64 if prec == 64 else torch.float32
    Xt = torch.from_numpy(Xv).to("cuda", dt).contiguous()
    Yt = torch.from_numpy(Yin).to("cuda", dt).contiguous()
    Ht.matmul(Xt, out=Yt, prec=prec, alpha=0.5, gamma=-0.25, beta=-1.0, Yin=Yt,
              Q=torch.from_numpy(Q).cuda(), hot_shift=10.0)
    tol = (TOL64 if prec == 64 else TOL32) * abs(Hfull).max() * np.abs(Xv).max() * 50
    assert np.abs(Yt.double().cpu().numpy() - ref).max() <= tol


@pytest.mark.parametrize("name", ["near_cutoff", "globule400"])
def test_store_matches_reference_dense_hessian(name):
    """The CUDA store (FP64 pair entries and, through products, the band tiles)
    against the reference's own dense Hessian X_D_K_Hessian (Burn/Coordinate/
    T3.py:47-127), stored by tests/golden/make_golden.py: 1e-12 of its largest entry."""
    from inching_b200.hessian import HessianStore
    g = np.load(f"tests/golden/hessian_{name}.npz")
    n = int(g["n"])
    L = np.zeros((n, n))
    L[g["rows"], g["cols"]] = g["vals"]
    Href = L + np.tril(L, -1).T
    H = HessianStore(g["X"], float(g["rc_nm"]) * 10.0, plus_i=float(g["plus_i"]), tiles=True)
    Lh = H.to_scipy_lower().toarray()
    Hs = Lh + np.tril(Lh, -1).T
    scale = np.abs(Href).max()
    assert np.abs(Hs - Href).max() <= TOL64 * scale
    # products through the band tiles: H e_k for a block of unit vectors = columns of Href
    E = torch.zeros((n, 40), dtype=torch.float64, device="cuda")
    cols = np.arange(0, n, max(1, n // 40))[:40]
    E[torch.from_numpy(cols).cuda(), torch.arange(len(cols), device="cuda")] = 1.0
    Y = H.matmul(E).cpu().numpy()
    assert np.abs(Y[:, :len(cols)] - Href[:, cols]).max() <= TOL64 * scale


@pytest.mark.parametrize("n", [1, 2, 5, 9, 33])
@pytest.mark.parametrize("prec", [64, 32])
def test_tiny_stores_every_width_and_traversal(n, prec):
    """Stores smaller than one row chunk, with an isolated atom and a coincident
    pair: every tile width (1 .. 130 columns) and every row traversal of the wide
    kernel gives the oracle's product."""
    from inching_b200 import _native
    from inching_b200.hessian import HessianStore
    rng = np.random.default_rng(n)
    X = rng.random((n, 3)) * 1.2
    if n >= 5:
        X[-1] = X[-1] + 5.0          # isolated atom
        X[1] = X[0]                  # coincident pair (d = 0: no spring)
    A, Ad = oh.hessian_lower(X, 8.0, 1.0)
    H = HessianStore(X, 8.0, plus_i=1.0)
    scale = max(float(abs(oh.full_from_lower(A, Ad)).max()), 1.0)
    dt = torch.float64 if prec == 64 else torch.float32
    try:
        for trav in (0, 1, 2):
            _native.spmm_tune(256, 5, trav)
            for b in (1, 3, 8, 64, 128, 130):
                Xv = rng.standard_normal((3 * n, b))
                ref = np.stack([oh.krylov_av(A, Ad, Xv[:, c]) for c in range(b)], axis=1)
                Y = H.matmul(torch.from_numpy(Xv).to("cuda", dt).contiguous(), prec=prec)
                tol = (TOL64 if prec == 64 else TOL32) * scale * np.abs(Xv).max() * 10
                assert np.abs(Y.double().cpu().numpy() - ref).max() <= tol, (trav, b)
    finally:
        _native.spmm_tune(256, 5, 1)
