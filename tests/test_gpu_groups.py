"""GPU parity of the row-group product (2 or 4 consecutive rows merged over their
neighbour lists, FP32) against the pair-layout kernel and the FP64 oracle
(restatement of Krylov/T3.py:128-160, Orthogonalization/T3.py:62-164,
PolynomialFilters/T2.py:59-80).

Each row of a group sums its own entries in the pair layout's order (zero-weight
slots in between add exact zeros), the order of the pair layout's wide kernel
(tiles of >= 8 columns; its narrower tiles split a row's entries over lanes).  So
without deflation, at widths that are multiples of 8, the group product is
compared with the pair kernel for bit equality, over every tile width (128 / 64
float4 / float2 tiles, 32-column tiles, partial last tiles), every in-flight
setting, unaligned blocks, the per-segment epilogue, periodic images (repeated
columns in a row), per-pair springs and stores smaller than one group.  With
Hotelling deflation the coefficient sums may be grouped differently per tile, so
those compare within FP32 rounding (2e-6 relative to ||H|| |X|, times a small
factor for the number of terms), as do the comparisons with the oracle."""
import numpy as np
import pytest
import torch

from oracle import hessian as oh

pytestmark = pytest.mark.gpu

TOL32 = 2e-6


@pytest.fixture(scope="module")
def case():
    from inching_b200 import graph, synth
    from inching_b200.hessian import HessianStore
    X = synth.globule(1500, seed=7) / 10.0
    order, _ = graph.cuthill_mckee(X, 8.0)
    Xr = X[order.cpu().numpy()]
    H = HessianStore(Xr, 8.0, plus_i=1.0)
    A, Ad = oh.hessian_lower(Xr, 8.0, 1.0)
    scale = float(abs(oh.full_from_lower(A, Ad)).max())
    return Xr, H, A, Ad, scale


def _stores(H):
    from inching_b200 import _native
    ent, _ = H.store(32)
    return {R: _native.group_store(H.rowptr, ent, H.n_atoms, R) for R in (2, 4)}


def _pair(H, X, Y=None, **kw):
    from inching_b200 import _native
    ent, diag = H.store(32)
    Y = torch.empty_like(X) if Y is None else Y
    b = X.shape[1]
    for c0 in range(0, b, 128):
        sl = slice(c0, min(c0 + 128, b))
        k = {key: (v[:, sl] if key in ("Yin", "acc") and v is not None else v) for key, v in kw.items()}
        _native.spmm(32, H.n_atoms, H.rowptr, ent, diag, X[:, sl], Y[:, sl], **k)
    return Y


def _same(Yg, Yp):
    """Bit equality where the pair kernel ran only wide tiles (b % 8 == 0), else
    agreement within FP32 rounding of the differently ordered sums."""
    if Yg.shape[-1] % 8 == 0:
        return torch.equal(Yg, Yp)
    return float((Yg - Yp).abs().max()) <= 1e-5 * (float(Yp.abs().max()) + 1.0)


def _merge_reference(rowptr, cols, ent, n, R, pad=16):
    """Host restatement of the group store: per group, the R-way merge of the rows'
    entry lists by column (rows advance together on equal heads), padded with
    zero-weight unions whose column is the group's first atom."""
    gcols, gw, gptr = [], [], [0]
    for g in range((n + R - 1) // R):
        rows = [r for r in range(R * g, min(R * g + R, n))]
        pos = {r: int(rowptr[r]) for r in rows}
        cnt = 0
        while True:
            heads = {r: int(cols[pos[r]]) for r in rows if pos[r] < rowptr[r + 1]}
            if not heads:
                break
            m = min(heads.values())
            slot = np.zeros((R, 3), dtype=np.float32)
            for r, h in heads.items():
                if h == m:
                    slot[r - R * g] = ent[pos[r], :3]
                    pos[r] += 1
            gcols.append(m)
            gw.append(slot)
            cnt += 1
        while cnt % pad:
            gcols.append(R * g)
            gw.append(np.zeros((R, 3), dtype=np.float32))
            cnt += 1
        gptr.append(gptr[-1] + cnt)
    return np.array(gptr), np.array(gcols), np.array(gw)


@pytest.mark.parametrize("R", [2, 4])
def test_group_store_layout_matches_host_merge(case, R):
    from inching_b200 import _native
    Xr, H, A, Ad, scale = case
    ent, _ = H.store(32)
    gptr, gent, nu = _native.group_store(H.rowptr, ent, H.n_atoms, R)
    rp = H.rowptr.cpu().numpy()
    cl = H.cols.cpu().numpy()
    e = ent.cpu().numpy()
    gp_ref, gc_ref, gw_ref = _merge_reference(rp, cl, e, H.n_atoms, R)
    assert np.array_equal(gptr.cpu().numpy(), gp_ref) and nu == gp_ref[-1]
    g = gent.cpu().numpy().reshape(nu, R, 4)
    assert np.array_equal(g[:, 0, 3].view(np.int32), gc_ref)
    assert np.array_equal(g[:, :, :3], gw_ref)
    assert (g[:, 1:, 3] == 0).all()


@pytest.mark.parametrize("b", [1, 5, 31, 32, 33, 64, 96, 100, 128, 129, 200, 320])
@pytest.mark.parametrize("R", [2, 4])
def test_group_product_matches_pair_kernel(case, R, b):
    from inching_b200 import _native
    Xr, H, A, Ad, scale = case
    gptr, gent, nu = _stores(H)[R]
    _, diag = H.store(32)
    g = torch.Generator(device="cuda")
    g.manual_seed(b)
    X = torch.randn((H.shape[0], b), generator=g, dtype=torch.float32, device="cuda")
    Yg = torch.full_like(X, float("nan"))
    _native.spmm_groups(H.n_atoms, R, gptr, gent, diag, X, Yg)
    assert _same(Yg, _pair(H, X))


@pytest.mark.parametrize("unroll", [0, 2, 4, 8, 16])
@pytest.mark.parametrize("R", [2, 4])
def test_group_in_flight_settings_same_bits(case, R, unroll):
    """The autotuner's in-flight setting changes the launch, not the product."""
    from inching_b200 import _native
    Xr, H, A, Ad, scale = case
    gptr, gent, nu = _stores(H)[R]
    _, diag = H.store(32)
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    X = torch.randn((H.shape[0], 224), generator=g, dtype=torch.float32, device="cuda")
    Yg = torch.empty_like(X)
    try:
        _native.spmm_group_tune(unroll)
        _native.spmm_groups(H.n_atoms, R, gptr, gent, diag, X, Yg)
    finally:
        _native.spmm_group_tune(0)
    assert torch.equal(Yg, _pair(H, X))


@pytest.mark.parametrize("b", [64, 128, 200])
def test_store_product_uses_groups_and_matches_oracle(case, b):
    """HessianStore.matmul runs FP32 products of >= 64 columns on the row groups
    (the remainder of a 64-column multiple on the pair kernel) and gives the
    oracle's Krylov product."""
    Xr, H, A, Ad, scale = case
    assert H.groups is not None and H._grouped(32, b) and not H._grouped(32, 63) and not H._grouped(64, b)
    rng = np.random.default_rng(b)
    Xv = rng.standard_normal((H.shape[0], b))
    ref = np.stack([oh.krylov_av(A, Ad, Xv[:, c]) for c in range(b)], axis=1)
    Y = H.matmul(torch.from_numpy(Xv).float().cuda().contiguous(), prec=32)
    assert np.abs(Y.double().cpu().numpy() - ref).max() <= TOL32 * scale * np.abs(Xv).max() * 10


@pytest.mark.parametrize("R", [2, 4])
@pytest.mark.parametrize("b", [40, 128, 136])
def test_group_fused_epilogue(case, R, b):
    """Y = a*HX + g*X + b*Yin + s*Q^T Q X (Yin aliasing Y) and Acc += mu*Y in one call:
    bit-equal to the pair kernel without deflation, within FP32 rounding with it."""
    from inching_b200 import _native
    Xr, H, A, Ad, scale = case
    gptr, gent, nu = _stores(H)[R]
    _, diag = H.store(32)
    rng = np.random.default_rng(b + R)
    Xv = rng.standard_normal((H.shape[0], b)).astype(np.float32)
    Yin = rng.standard_normal((H.shape[0], b)).astype(np.float32)
    Acc0 = rng.standard_normal((H.shape[0], b)).astype(np.float32)
    Q = oh.rigid_body_basis(Xr)
    a, gm, be, s, mu = 0.37, -1.25, -1.0, 10.0, 0.6
    t = lambda m: torch.from_numpy(m).cuda().contiguous()
    Xt = t(Xv)
    for with_q in (False, True):
        kw = dict(alpha=a, gamma=gm, beta=be, mu=mu)
        if with_q:
            kw.update(Q=torch.from_numpy(Q).cuda(), hot_shift=s)
        Yg, Accg = t(Yin), t(Acc0)
        _native.spmm_groups(H.n_atoms, R, gptr, gent, diag, Xt, Yg, Yin=Yg, acc=Accg, **kw)
        Yp, Accp = t(Yin), t(Acc0)
        _pair(H, Xt, Yp, Yin=Yp, acc=Accp, **kw)
        if not with_q:
            assert torch.equal(Yg, Yp) and torch.equal(Accg, Accp)
        else:
            ref = (a * np.stack([oh.krylov_av(A, Ad, Xv[:, c].astype(np.float64)) for c in range(b)], axis=1)
                   + gm * Xv + be * Yin + s * Q.T @ (Q @ Xv.astype(np.float64)))
            tol = TOL32 * scale * 50 * np.abs(Xv).max()
            assert np.abs(Yg.double().cpu().numpy() - ref).max() <= tol
            assert np.abs(Accg.double().cpu().numpy() - (Acc0 + mu * ref)).max() <= tol
            assert float((Yg - Yp).abs().max()) <= tol


def test_group_unaligned_blocks_and_untouched_columns(case):
    """Odd leading dimension and column offset: the group product runs 32-column
    tiles (no vector access, the last one partial), gives the pair kernel's bits,
    and leaves the columns
    outside the view untouched."""
    from inching_b200 import _native
    Xr, H, A, Ad, scale = case
    gptr, gent, nu = _stores(H)[2]
    _, diag = H.store(32)
    b, ld = 72, 75
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    Xt = torch.randn((H.shape[0], ld), generator=g, dtype=torch.float32, device="cuda")
    Yt = torch.zeros_like(Xt)
    _native.spmm_groups(H.n_atoms, 2, gptr, gent, diag, Xt[:, 1:1 + b], Yt[:, 1:1 + b])
    Yp = torch.zeros_like(Xt)
    _native.spmm(32, H.n_atoms, H.rowptr, H.ent32, diag, Xt[:, 1:1 + b], Yp[:, 1:1 + b])
    assert torch.equal(Yt, Yp)
    assert float(Yt[:, 0].abs().max()) == 0.0 and float(Yt[:, 1 + b:].abs().max()) == 0.0


@pytest.mark.parametrize("R", [2, 4])
def test_group_segmented_matches_pair_kernel(case, R):
    """Per-segment (alpha, gamma, beta) on the row groups equals the pair kernel's."""
    from inching_b200 import _native
    Xr, H, A, Ad, scale = case
    gptr, gent, nu = _stores(H)[R]
    ent, diag = H.store(32)
    n, b = H.n_atoms, 160
    seg = torch.zeros(n, dtype=torch.int32, device="cuda")
    seg[n // 3:] = 1
    coef = torch.tensor([[0.5, -0.2, -1.0], [2.0, 0.3, 0.25]], dtype=torch.float64, device="cuda")
    g = torch.Generator(device="cuda")
    g.manual_seed(4)
    X = torch.randn((3 * n, b), generator=g, dtype=torch.float32, device="cuda")
    Yin = torch.randn((3 * n, b), generator=g, dtype=torch.float32, device="cuda")
    Y1 = torch.empty_like(X)
    _native.spmm_groups_seg(n, R, gptr, gent, diag, X, Y1, seg, coef, Yin=Yin)
    Y2 = torch.empty_like(X)
    for c0 in range(0, b, 128):
        sl = slice(c0, min(c0 + 128, b))
        _native.spmm_seg(32, n, H.rowptr, ent, diag, X[:, sl], Y2[:, sl], seg, coef, Yin=Yin[:, sl])
    assert torch.equal(Y1, Y2)
    Y3 = torch.empty_like(X)
    H.matmul_seg(X, Y3, seg, coef, Yin=Yin, prec=32)           # the store's own path (groups + remainder)
    assert torch.equal(Y3, Y2)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 9])
def test_group_tiny_stores(n):
    """Stores smaller than a group or with a partial last group, an isolated atom
    and a coincident pair: every tile width gives the pair kernel's product."""
    from inching_b200 import _native
    from inching_b200.hessian import HessianStore
    rng = np.random.default_rng(n)
    X = rng.random((n, 3)) * 1.2
    if n >= 5:
        X[-1] = X[-1] + 5.0
        X[1] = X[0]
    H = HessianStore(X, 8.0, plus_i=1.0)
    _, diag = H.store(32)
    for R in (2, 4):
        gptr, gent, nu = _native.group_store(H.rowptr, H.ent32, n, R)
        for b in (1, 3, 32, 64, 128, 130):
            Xv = torch.from_numpy(rng.standard_normal((3 * n, b))).float().cuda().contiguous()
            Yg = torch.empty_like(Xv)
            _native.spmm_groups(n, R, gptr, gent, diag, Xv, Yg)
            assert _same(Yg, _pair(H, Xv)), (R, b)


def test_group_periodic_and_weighted_stores():
    """Periodic xy images (a row may hold one column twice, through two images) and
    per-pair springs: the group store copies the pair entries, so the product keeps
    the pair kernel's bits."""
    import os
    from conftest import GOLDEN
    from inching_b200 import _native, synth
    from inching_b200.hessian import HessianStore
    gz = np.load(os.path.join(GOLDEN, "pbc_slab.npz"))
    box = gz["box"]
    d = {"RectBox_Xsize": box[0], "RectBox_Ysize": box[1], "RectBox_Zsize": box[2],
         "X": (0.0, box[0]), "Y": (0.0, box[1]), "Z": (0.0, box[2])}
    stores = [HessianStore(gz["X"], 8.0, 1.0, pbc=d)]
    Xw = synth.globule(800, seed=3) / 10.0
    Hw0 = HessianStore(Xw, 8.0, 1.0)
    rows = torch.repeat_interleave(torch.arange(Hw0.n_atoms, device="cuda"), torch.diff(Hw0.rowptr))
    key = (torch.minimum(rows, Hw0.cols.long()) * 7919 + torch.maximum(rows, Hw0.cols.long())).double()
    gam = 0.5 + (torch.sin(key * 0.37) + 1.0)
    stores.append(HessianStore(Xw, 8.0, 1.0, graph_=(Hw0.degree, Hw0.rowptr, Hw0.cols), pair_weight=gam))
    for H in stores:
        assert H.groups is not None
        g = torch.Generator(device="cuda")
        g.manual_seed(2)
        X = torch.randn((H.shape[0], 128), generator=g, dtype=torch.float32, device="cuda")
        Yg = H.matmul(X, prec=32)
        assert torch.equal(Yg, _pair(H, X))


def test_group_at_scale_matches_pair_kernel():
    """100,000-atom assembly: the group product (both group sizes) gives the pair
    kernel's bits on 320 columns, and the six rigid-body vectors stay eigenvectors
    (H q = PlusI q) through it within FP32 rounding."""
    from inching_b200 import _native, graph, synth
    from inching_b200.hessian import HessianStore
    X = synth.workload("assembly100k") / 10.0
    order, _ = graph.cuthill_mckee(X, 8.0)
    Xr = X[order.cpu().numpy()]
    H = HessianStore(Xr, 8.0, plus_i=1.0, precisions=("f32",))
    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    Xp = torch.randn((H.shape[0], 320), generator=g, dtype=torch.float32, device="cuda")
    ref = _pair(H, Xp)
    _, diag = H.store(32)
    for R in (2, 4):
        gptr, gent, nu = _native.group_store(H.rowptr, H.ent32, H.n_atoms, R)
        Y = torch.empty_like(Xp)
        _native.spmm_groups(H.n_atoms, R, gptr, gent, diag, Xp, Y)
        assert torch.equal(Y, ref), R
        assert H.nnz_blocks / nu > 1.2          # unions shared by the group's rows
    Q = torch.from_numpy(oh.rigid_body_basis(Xr).T.copy()).float().cuda()
    Qp = torch.zeros((H.shape[0], 64), dtype=torch.float32, device="cuda")
    Qp[:, :6] = Q
    Y = H.matmul(Qp, prec=32)
    assert float((Y[:, :6] - Q).abs().max()) < 1e-4
