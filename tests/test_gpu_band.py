"""GPU parity of the band-tile product (8-row tiles, union walk) against the FP64
oracle (restatement of Krylov/T3.py:128-160, Orthogonalization/T3.py:62-164,
PolynomialFilters/T2.py:59-80) and against the pair-layout kernel.

Every panel width of the kernel is reached: FP32 panels of 128 (packed f32x2),
64 and 32 columns, FP64 panels of 64 and 32, partial last panels, unaligned
leading dimensions (scalar panels), single vectors when the pair entries are
dropped, the fused epilogue (shift, three-term step with Yin aliasing Y,
accumulation, Hotelling deflation) and the per-segment coefficients.

Tolerances: FP64 1e-12 relative to ||H|| |X|; FP32 2e-6 relative to ||H|| |X|
(single-precision rounding of w and of the sums), both times a small factor for
the number of terms."""
import numpy as np
import pytest
import torch

from oracle import hessian as oh

pytestmark = pytest.mark.gpu

TOL = {64: 1e-12, 32: 2e-6}


@pytest.fixture(scope="module")
def case():
    from inching_b200 import graph, synth
    from inching_b200.hessian import HessianStore
    X = synth.globule(1500, seed=7) / 10.0
    order, _ = graph.cuthill_mckee(X, 8.0)
    Xr = X[order.cpu().numpy()]
    H = HessianStore(Xr, 8.0, plus_i=1.0, tiles=True)
    A, Ad = oh.hessian_lower(Xr, 8.0, 1.0)
    scale = float(abs(oh.full_from_lower(A, Ad)).max())
    Q = oh.rigid_body_basis(Xr)
    return Xr, H, A, Ad, scale, Q


def _ref(A, Ad, Xv):
    return np.stack([oh.krylov_av(A, Ad, Xv[:, c]) for c in range(Xv.shape[1])], axis=1)


@pytest.mark.parametrize("b", [8, 24, 32, 40, 64, 96, 128, 136, 200, 320])
@pytest.mark.parametrize("prec", [64, 32])
def test_band_product_matches_krylov_av(case, prec, b):
    Xr, H, A, Ad, scale, Q = case
    assert H._tiled(prec, b)
    rng = np.random.default_rng(b)
    Xv = rng.standard_normal((H.shape[0], b))
    ref = _ref(A, Ad, Xv)
    dt = torch.float64 if prec == 64 else torch.float32
    Y = H.matmul(torch.from_numpy(Xv).to("cuda", dt).contiguous(), prec=prec)
    tol = TOL[prec] * scale * np.abs(Xv).max() * 10
    assert np.abs(Y.double().cpu().numpy() - ref).max() <= tol


@pytest.mark.parametrize("widest", [128, 64])
@pytest.mark.parametrize("prec", [64, 32])
def test_band_launch_choice_same_product(case, widest, prec):
    """The autotuner's switch (128- or 64-column FP32 panels) changes the launch
    shape, not the product."""
    from inching_b200 import _native
    Xr, H, A, Ad, scale, Q = case
    rng = np.random.default_rng(5)
    Xv = rng.standard_normal((H.shape[0], 200))
    ref = _ref(A, Ad, Xv)
    dt = torch.float64 if prec == 64 else torch.float32
    try:
        _native.spmm_band_tune(widest)
        Y = H.matmul(torch.from_numpy(Xv).to("cuda", dt).contiguous(), prec=prec)
    finally:
        _native.spmm_band_tune(128)
    assert np.abs(Y.double().cpu().numpy() - ref).max() <= TOL[prec] * scale * np.abs(Xv).max() * 10


@pytest.mark.parametrize("prec", [64, 32])
@pytest.mark.parametrize("b", [40, 128, 136])
def test_band_fused_epilogue(case, prec, b):
    """Y = a*HX + g*X + b*Yin + s*Q^T Q X (Yin aliasing Y) and Acc += mu*Y in one call."""
    Xr, H, A, Ad, scale, Q = case
    rng = np.random.default_rng(b + prec)
    Xv = rng.standard_normal((H.shape[0], b))
    Yin = rng.standard_normal((H.shape[0], b))
    Acc0 = rng.standard_normal((H.shape[0], b))
    a, g, be, s, mu = 0.37, -1.25, -1.0, 10.0, 0.6
    ref = a * _ref(A, Ad, Xv) + g * Xv + be * Yin + s * Q.T @ (Q @ Xv)
    dt = torch.float64 if prec == 64 else torch.float32
    t = lambda m: torch.from_numpy(m).to("cuda", dt).contiguous()
    Xt, Yt, Acc = t(Xv), t(Yin), t(Acc0)
    H.matmul(Xt, out=Yt, prec=prec, alpha=a, gamma=g, beta=be, Yin=Yt, acc=Acc, mu=mu,
             Q=torch.from_numpy(Q).cuda(), hot_shift=s)
    tol = TOL[prec] * scale * 50 * np.abs(Xv).max()
    assert np.abs(Yt.double().cpu().numpy() - ref).max() <= tol
    assert np.abs(Acc.double().cpu().numpy() - (Acc0 + mu * ref)).max() <= tol


@pytest.mark.parametrize("prec", [64, 32])
def test_band_unaligned_leading_dimension(case, prec):
    """Odd leading dimension and column offset: the C ABI refuses the block (its
    rows are staged as 16-byte bulk copies), the store's product pads it and gives
    the same result, and the columns outside the view stay untouched."""
    from inching_b200 import _native
    Xr, H, A, Ad, scale, Q = case
    b, ld = 70, 73
    rng = np.random.default_rng(11)
    Xv = rng.standard_normal((H.shape[0], ld))
    ref = _ref(A, Ad, Xv[:, 1:1 + b])
    dt = torch.float64 if prec == 64 else torch.float32
    Xt = torch.from_numpy(Xv).to("cuda", dt)
    Yt = torch.zeros_like(Xt)
    t = H.tiles
    _, diag = H.store(prec)
    with pytest.raises(AssertionError, match="ABORTED"):
        _native.spmm_tiles(prec, H.n_atoms, t["uptr"], t["pptr"], t["urec"], t["pw64" if prec == 64 else "pw32"],
                           diag, Xt[:, 1:1 + b], Yt[:, 1:1 + b])
    H.matmul(Xt[:, 1:1 + b], out=Yt[:, 1:1 + b], prec=prec, alpha=1.0, gamma=0.0)
    tol = TOL[prec] * scale * np.abs(Xv).max() * 10
    assert np.abs(Yt[:, 1:1 + b].double().cpu().numpy() - ref).max() <= tol
    assert float(Yt[:, 0].abs().max()) == 0.0 and float(Yt[:, 1 + b:].abs().max()) == 0.0
    assert _native.spmm_band_status() == 0


@pytest.mark.parametrize("prec", [64, 32])
def test_band_only_store_single_vector(case, prec):
    """keep_pairs=False: the pair entries are dropped and every product, single
    vectors included, runs on the band tiles."""
    from inching_b200.hessian import HessianStore
    Xr, H, A, Ad, scale, Q = case
    Hb = HessianStore(Xr, 8.0, plus_i=1.0, tiles=True, keep_pairs=False)
    assert Hb.ent64.numel() == 0 and Hb.ent32.numel() == 0
    rng = np.random.default_rng(2)
    v = rng.standard_normal(H.shape[0])
    dt = torch.float64 if prec == 64 else torch.float32
    y = Hb.matmul(torch.from_numpy(v).to("cuda", dt), prec=prec)
    ref = oh.krylov_av(A, Ad, v)
    assert np.abs(y.double().cpu().numpy() - ref).max() <= TOL[prec] * scale * np.abs(v).max() * 10
    Xv = rng.standard_normal((H.shape[0], 3))
    Y = Hb.matmul(torch.from_numpy(Xv).to("cuda", dt).contiguous(), prec=prec)
    assert np.abs(Y.double().cpu().numpy() - _ref(A, Ad, Xv)).max() <= TOL[prec] * scale * np.abs(Xv).max() * 10


@pytest.mark.parametrize("prec", [64, 32])
def test_band_segmented_matches_pair_kernel(case, prec):
    """Per-segment (alpha, gamma, beta) on the band tiles equals the pair kernel's."""
    from inching_b200 import _native
    Xr, H, A, Ad, scale, Q = case
    b = 96
    n = H.n_atoms
    seg = torch.zeros(n, dtype=torch.int32, device="cuda")
    seg[n // 2:] = 1
    coef = torch.tensor([[0.5, -0.2, -1.0], [2.0, 0.3, 0.25]], dtype=torch.float64, device="cuda")
    dt = torch.float64 if prec == 64 else torch.float32
    g = torch.Generator(device="cuda")
    g.manual_seed(4)
    X = torch.randn((3 * n, b), generator=g, dtype=torch.float64, device="cuda").to(dt)
    Yin = torch.randn((3 * n, b), generator=g, dtype=torch.float64, device="cuda").to(dt)
    Y1 = torch.empty_like(X)
    H.matmul_seg(X, Y1, seg, coef, Yin=Yin, prec=prec)
    Y2 = torch.empty_like(X)
    ent, diag = H.store(prec)
    for c0 in range(0, b, 32):
        sl = slice(c0, c0 + 32)
        _native.spmm_seg(prec, n, H.rowptr, ent, diag, X[:, sl], Y2[:, sl], seg, coef, Yin=Yin[:, sl])
    tol = TOL[prec] * scale * 20 * float(X.abs().max())
    assert float((Y1.double() - Y2.double()).abs().max()) <= tol


def test_band_at_scale_matches_pair_kernel():
    """100,000-atom assembly: the band product equals the pair kernel's on 320
    columns (FP32 and FP64), and the six rigid-body vectors stay exact
    eigenvectors (H q = PlusI q) through the band tiles."""
    from inching_b200 import graph, synth
    from inching_b200.hessian import HessianStore
    X = synth.workload("assembly100k") / 10.0
    order, _ = graph.cuthill_mckee(X, 8.0)
    Xr = X[order.cpu().numpy()]
    H = HessianStore(Xr, 8.0, plus_i=1.0, tiles=True)
    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    X64 = torch.randn((H.shape[0], 320), generator=g, dtype=torch.float64, device="cuda")
    for prec, tol in ((64, 1e-12), (32, 2e-6)):
        Xp = X64 if prec == 64 else X64.float()
        Yb = H.matmul(Xp.contiguous(), prec=prec)
        H.use_tiles = False
        try:
            Yp = H.matmul(Xp.contiguous(), prec=prec)
        finally:
            H.use_tiles = True
        ref = float(Yp.double().abs().max())
        assert float((Yb.double() - Yp.double()).abs().max()) <= tol * 10 * ref
    Q = torch.from_numpy(oh.rigid_body_basis(Xr).T.copy()).cuda()
    Qp = torch.zeros((H.shape[0], 8), dtype=torch.float64, device="cuda")
    Qp[:, :6] = Q
    Y = H.matmul(Qp, prec=64)
    assert float((Y[:, :6] - Q).abs().max()) < 1e-11
