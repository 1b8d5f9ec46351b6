"""Host-side logic of the solvers, on CPU: the degree and guard rules, the filter
coefficient tables, the periodic-box parser, and the control flow of the
per-column filter and of the Chebyshev-Davidson and block solvers run against a
dense CPU test double of the Hessian store (the product itself needs CUDA)."""
import numpy as np
import pytest
import torch

from oracle import hessian as oh


class DenseStore:
    """Test double with the store's matmul interface (fused epilogue) on a dense
    CPU matrix."""

    def __init__(self, H):
        self.Hd = torch.from_numpy(np.asarray(H))
        self.shape = self.Hd.shape
        self.device = torch.device("cpu")
        self.ndim = 2
        self.dtype = torch.float64

    def matmul(self, X, out=None, prec=64, alpha=1.0, gamma=0.0, beta=0.0, Yin=None, acc=None, mu=0.0, Q=None,
               hot_shift=0.0):
        H = self.Hd.to(X.dtype)
        Y = alpha * (H @ X) + gamma * X
        if Yin is not None:
            Y = Y + beta * Yin
        if Q is not None and hot_shift:
            q = Q.to(X.dtype)
            Y = Y + hot_shift * (q.t() @ (q @ X))
        if acc is not None:
            acc += mu * Y
        if out is not None:
            out.copy_(Y)
            return out
        return Y


@pytest.fixture(scope="module")
def dense():
    from inching_b200 import synth
    X = synth.globule(300, seed=3) / 10.0
    A, Ad = oh.hessian_lower(X, 8.0, 1.0)
    H = oh.full_from_lower(A, Ad).toarray()
    w, U = np.linalg.eigh(H)
    Q = torch.from_numpy(oh.rigid_body_basis(X))
    return dict(F=DenseStore(H), w=w, U=U, Q=Q)


def test_lean_degree_rule():
    from inching_b200.solvers.chfsi import lean_degree

    class S:
        pass

    def deg(n_atoms, nnz, p):
        a = S()
        a.shape = (3 * n_atoms, 3 * n_atoms)
        a.nnz_blocks = nnz
        return lean_degree(a, p)

    assert deg(100000, 10064346, 320) == 24          # the 100k-atom configuration
    assert deg(2400000, 241e6, 1250) == 48           # 1,000 modes of 2.4M atoms
    assert deg(498000, 51e6, 1250) == 48
    assert deg(10**7, 1e9, 5000) == 64               # capped
    assert lean_degree(S(), 100) == 24               # an operator without a block count


def test_batched_guard_rounds_to_panels():
    from inching_b200.solvers.batched import batched_guard
    assert batched_guard(32) == 32 and (32 + batched_guard(32)) % 32 == 0
    for k in (1, 8, 12, 33, 64, 100):
        g = batched_guard(k)
        assert g >= max(16, int(np.ceil(k / 2))) and (k + g) % 32 == 0


def test_chebyshev_degrees():
    from inching_b200.solvers.chfsi import chebyshev_degrees
    theta = np.array([1.2, 2.0, 4.9, 5.0, 7.0])
    res = np.array([1e-3, 1e-5, 1e-2, 1.0, 1.0])
    d = chebyshev_degrees(theta, res, 3, 1e-6, 5.0, 60.0, 24)
    assert list(d[3:]) == [24, 24]                    # guard vectors keep the full degree
    assert d[1] < d[0] <= 24 and d[2] == 24           # closer to converged, further from a: fewer steps
    assert (d >= 2).all()


def test_cdm_filter_rows_are_chebyshev():
    from inching_b200.solvers.cdm import filter_rows
    low, high, m = 3.0, 40.0, 9
    rows = filter_rows(m, low, high)
    e, c = (high - low) / 2, (high + low) / 2
    for lam in (0.5, 2.9, 10.0, 39.0):
        x0 = 1.0
        a0, g0, _ = rows[0]
        x1 = a0 * lam * x0 + g0 * x0
        prev, cur = x0, x1
        for a, g, b in rows[1:]:
            prev, cur = cur, a * lam * cur + g * cur + b * prev
        ref = np.polynomial.chebyshev.chebval((c - lam) / e, [0] * (m + 1) + [1])
        assert cur == pytest.approx(ref, rel=1e-10)


def test_pbc_box_parser():
    from inching_b200.graph import pbc_box
    assert pbc_box(None) is None
    assert pbc_box({"RectBox_Xsize": 3.5, "RectBox_Ysize": 2.0, "RectBox_Zsize": 9.0}) == (3.5, 2.0)
    assert pbc_box((1, 2)) == (1.0, 2.0)


def test_per_column_filter_equals_single_degree_runs(dense):
    from inching_b200.solvers.chfsi import _Filter
    f = _Filter(dense["F"], 64)
    X = torch.randn(dense["F"].shape[0], 13, dtype=torch.float64, generator=torch.Generator().manual_seed(1))
    degs = np.random.default_rng(0).integers(1, 10, size=13)
    a, b, a0 = 5.0, dense["w"][-1] * 1.02, dense["w"][0]
    Z = f(X, 9, a, b, a0, degrees=degs)
    for i in range(13):
        zi = f(X[:, i:i + 1].contiguous(), int(degs[i]), a, b, a0)
        assert torch.allclose(zi[:, 0], Z[:, i], rtol=0, atol=1e-12 * float(zi.abs().max()))


@pytest.mark.parametrize("block,with_q", [(1, False), (1, True), (4, True)])
def test_cdm_control_flow_on_dense_double(dense, block, with_q):
    from inching_b200.solvers.cdm import cdm
    w = dense["w"]
    S, V, info = cdm(dense["F"], 12, tol=1e-10, degree=12, spectrum_bound=(w[0], w[-1]), cuda_graph=False,
                     Q=dense["Q"] if with_q else None, block=block, return_info=True)
    off = 6 if with_q else 0
    assert info["converged"]
    assert np.abs(S.numpy() - w[off:off + 12]).max() < 1e-9 * w[-1]


def test_block_solver_control_flow_on_dense_double(dense):
    from inching_b200.solvers.chfsi import chfsi
    w = dense["w"]
    S, V, info = chfsi(dense["F"], 20, tol=1e-9, Q=dense["Q"], precision="f64", return_info=True)
    assert info["converged"] and info["max_rel_residual"] <= 1.5e-9
    assert np.abs(S.numpy() - w[6:26]).max() < 1e-8 * w[-1]


@pytest.mark.parametrize("maxiter", [300, 1])
def test_block_solver_returns_whole_orthonormal_block(dense, maxiter):
    """return_block: the k locked modes followed by the guard's Ritz vectors, all
    orthonormal and orthogonal to the deflated rows, after a converged exit and
    after one that stopped at maxiter."""
    import torch
    from inching_b200.solvers.chfsi import chfsi
    w = dense["w"]
    S, B, info = chfsi(dense["F"], 20, tol=1e-9, Q=dense["Q"], precision="f64", guard=12, maxiter=maxiter,
                       return_block=True, return_info=True)
    assert B.shape == (dense["F"].shape[0], 32) and S.shape == (20,)
    assert info["converged"] == (maxiter == 300)
    eye = torch.eye(32, dtype=torch.float64)
    assert (B.t() @ B - eye).abs().max() < 1e-10
    Q = torch.as_tensor(dense["Q"], dtype=torch.float64)
    assert (Q @ B).abs().max() < 1e-10
    if info["converged"]:
        assert np.abs(S.numpy() - w[6:26]).max() < 1e-8 * w[-1]


@pytest.mark.parametrize("precision,tol,fold", [("f64", 1e-9, True), ("mixed", 1e-6, True), ("mixed", 1e-6, False)])
def test_lean_block_solver_chunked_paths_on_dense_double(dense, precision, tol, fold):
    """chfsi_lean with chunks smaller than the block (column chunks of the filter,
    row chunks of rotations and projections, a residual window shorter than the
    wanted count), and with a caller's FP64 block X0 of the full width taken over
    in place: the eigenvalues of the dense Hessian, orthonormal vectors; with the
    second Cholesky-QR pass's factor folded into the Rayleigh-Ritz rotation and
    with two full passes."""
    from inching_b200.solvers.chfsi import chfsi_lean, default_guard
    w = dense["w"]
    n, k = dense["F"].shape[0], 20
    X0 = torch.randn((n, k + default_guard(k)), generator=torch.Generator().manual_seed(1), dtype=torch.float64)
    S, V, info = chfsi_lean(dense["F"], k, tol=tol, Q=dense["Q"], precision=precision, chunk=16, row_chunk=256,
                            window=12, X0=X0, return_info=True, fold_orth=fold)
    assert info["converged"] and info["max_rel_residual"] <= 1.5 * tol
    assert np.abs(S.numpy() - w[6:26]).max() < (1e-8 if precision == "f64" else 1e-4) * w[-1]
    assert (V.t() @ V - torch.eye(k, dtype=V.dtype)).abs().max() < 1e-10
    assert (dense["Q"] @ V).abs().max() < 1e-10


@pytest.mark.parametrize("name,k,tol", [("trlm", 12, 1e-10), ("jdm", 12, 1e-8), ("irlm", 32, 1e-10)])
def test_reference_solver_control_flow_on_dense_double(dense, name, k, tol):
    """The reference algorithms' host control flow (TRLM thick restarts, JDM with
    its projected GMRES correction and locking, IRLM implicit restarts) with
    Hotelling deflation of the rigid modes, on the dense test double: the
    eigenvalues of dense LAPACK and orthonormal eigenvectors orthogonal to the
    rigid-body basis.  IRLM keeps the reference's refusal of fewer than 32 modes."""
    import importlib
    fn = getattr(importlib.import_module(f"inching_b200.solvers.{name}"), name)
    w = dense["w"]
    S, V = fn(dense["F"], k=k, tol=tol, Q=dense["Q"], shift=10.0)[:2]
    assert np.abs(S.numpy() - w[6:6 + k]).max() < 1e-10 * w[-1]
    assert (V.t() @ V - torch.eye(k, dtype=V.dtype)).abs().max() < 1e-8
    assert (dense["Q"] @ V).abs().max() < 1e-8
    if name == "irlm":
        with pytest.raises(AssertionError, match="ABORTED"):
            fn(dense["F"], k=16, tol=tol, Q=dense["Q"], shift=10.0)


def test_ctrlm_march_and_resume_on_dense_double(dense, tmp_path):
    """Interval marching on the dense double: one window written to the
    reference's window pickles, then a second call resumes from them.  Together
    the two calls find the 40 lowest non-rigid modes of dense LAPACK with no
    duplicate and no gap, and each window has its Eigval / PerformanceList file."""
    from inching_b200.ctrlm import ctrlm_many_modes
    F = dense["F"]
    F.plus_i, F.n_atoms = 1.0, F.shape[0] // 3
    w = dense["w"] - 1.0
    ck = dict(folder=str(tmp_path), pdbid="toy", platform="Linux", device="cpu")
    a = ctrlm_many_modes(F, 40, n_mode=16, Q=dense["Q"], tol=1e-10, checkpoint=ck, max_windows=1)
    assert not a["complete"] and len(a["windows"]) == 1
    b = ctrlm_many_modes(F, 40, n_mode=16, Q=dense["Q"], tol=1e-10, checkpoint=ck)
    assert b["complete"] and b["windows"][0]["offset"] == len(a["eigvals"])
    ev = np.sort(np.concatenate([a["eigvals"], b["eigvals"]]))
    assert len(ev) >= 40 and np.diff(ev).min() > 1e-6
    assert np.abs(ev[:40] - w[6:46]).max() < 1e-10 * w[-1]
    for win in a["windows"] + b["windows"]:
        for kind in ("Eigval", "PerformanceList"):
            assert (tmp_path / f"{kind}_InchingManyCTRLM_toy_Linux_cpu_{win['offset']}.pkl").exists()


def test_solver_facades_on_dense_double(dense):
    """The drop-in solver entry points with the reference's argument names
    (A, A_diag, k, tol, User_Q_HotellingDeflation, ...) return its layout:
    eigenvalues including PlusI and eigenvectors as (n, k) columns; and they
    keep the reference's refusals (JDM with a polynomial filter or a workspace
    factor <= 1, TRLM with k >= n)."""
    from inching_b200.Burn.ImplicitlyRestartedLanczosHotellingDeflation.T1 import S_HeigvalIRLMHD_HeigvecIRLMHD
    from inching_b200.Burn.JacobiDavidsonHotellingDeflation.T1 import S_HeigvalJDMHD_HeigvecJDMHD
    from inching_b200.Burn.ThickRestartLanczosHotellingDeflation.T1 import S_HeigvalTRLMHD_HeigvecTRLMHD
    F, Q, w = dense["F"], dense["Q"], dense["w"]
    Ad = torch.from_numpy(np.diag(F.Hd.numpy()).copy())
    n = F.shape[0]
    for S, V, k in ((*S_HeigvalTRLMHD_HeigvecTRLMHD(F, Ad, k=12, tol=1e-10, User_Q_HotellingDeflation=Q)[:2], 12),
                    (*S_HeigvalJDMHD_HeigvecJDMHD(F, Ad, k=12, tol=1e-8, User_Q_HotellingDeflation=Q)[:2], 12),
                    (*S_HeigvalIRLMHD_HeigvecIRLMHD(F, k=32, tol=1e-10, User_Q_HotellingDeflation=Q)[:2], 32)):
        assert tuple(V.shape) == (n, k)
        assert np.abs(np.sort(np.asarray(S.cpu())) - w[6:6 + k]).max() < 1e-10 * w[-1]
    with pytest.raises(AssertionError, match="ABORTED"):
        S_HeigvalJDMHD_HeigvecJDMHD(F, Ad, k=12, User_WorkspaceSizeFactor=1)
    with pytest.raises(AssertionError, match="ABORTED"):
        S_HeigvalJDMHD_HeigvecJDMHD(F, Ad, k=12, User_PolynomialParams=object())
    with pytest.raises(AssertionError, match="ABORTED"):
        S_HeigvalTRLMHD_HeigvecTRLMHD(F, Ad, k=n)


def test_operator_facades_against_oracle_on_dense_double(dense):
    """Krylov aux(A, v, u), the Hotelling update, ChebyshevAv (with the KPM rho)
    and the Lanczos spectrum bound through the drop-in module paths, against the
    oracle's restatements of Krylov/T3.py, Orthogonalization/T3.py and
    PolynomialFilters/T2.py on the dense test double."""
    from oracle import solvers as osv
    from inching_b200 import polyfilter
    from inching_b200.Burn.HermitianLanczos.T2 import A_Adiag_EstimateSpectrumBound
    from inching_b200.Burn.Krylov.T3 import OOC2_FullMemS_v_KrylovAv_VOID, OOC2_HalfMemS_v_KrylovAv_VOID
    from inching_b200.Burn.Orthogonalization.T3 import T3_QHotelling_x_Ax_HotelledAx
    from inching_b200.Burn.PolynomialFilters.T2 import OOC2_A_Adiag_ChebyshevAv
    F, Q, w = dense["F"], dense["Q"], dense["w"]
    Hd = F.Hd.numpy()
    Ad = torch.from_numpy(np.diag(Hd).copy())
    v = torch.from_numpy(np.random.default_rng(2).standard_normal(F.shape[0]))
    for factory in (OOC2_HalfMemS_v_KrylovAv_VOID, OOC2_FullMemS_v_KrylovAv_VOID):
        u = torch.empty_like(v)
        assert factory(F, Ad)(F, v, u) is None
        assert np.abs(u.numpy() - Hd @ v.numpy()).max() < 1e-12 * np.abs(Hd).max()
    res = torch.zeros_like(v)
    T3_QHotelling_x_Ax_HotelledAx(Q, v, res, HotellingShift=-40.0)
    ref = oh.hotelling(Q.numpy(), v.numpy(), np.zeros(F.shape[0]), -40.0)
    assert np.abs(res.numpy() - ref).max() < 1e-12 * np.abs(ref).max()
    lo, hi = A_Adiag_EstimateSpectrumBound(F, Ad)
    assert abs(hi - w[-1]) < 1e-6 * w[-1] and abs(lo - w[0]) < 1e-6 * w[-1]
    pol = polyfilter.OOC0_OptimizePolynomialParamsOnDegree(User_WantedInterval=(1.0, 3.0),
                                                           User_SpectrumBound=(0.99, w[-1] * 1.01),
                                                           User_MaximumDegree=300)
    ref = osv.chebyshev_av(lambda x: Hd @ x, v.numpy(), pol.AdjustedCoefficients, pol.cc, pol.dd, pol.AdjustedDegree)
    for precision, tol in (("f64", 1e-10), ("mixed", 1e-4)):
        y = OOC2_A_Adiag_ChebyshevAv(F, Ad, User_PolynomialParams=pol, User_Precision=precision).ChebyshevAv(F, v)
        assert np.abs(y.double().numpy() - ref).max() <= tol * np.abs(ref).max()
    with pytest.raises(AssertionError, match="ABORTED"):
        OOC2_A_Adiag_ChebyshevAv(F, Ad)


def test_cdm_and_kpm_facades_on_dense_double(dense):
    """Chebyshev-Davidson through the reference signature (no deflation: the six
    rigid modes at PlusI come first) against dense LAPACK, its three refusals, and
    the KPM eigenvalue count of a window within 30 % of the true count."""
    from inching_b200 import polyfilter
    from inching_b200.Burn.ChebyshevDavidsonSubspaceIteration.T1 import (OOC2_KrylovAv_A_EstimateSpectrumBound,
                                                                           S_HeigvalCDSIHD_HeigvecCDSIHD)
    from inching_b200.Burn.PolynomialFilters.T2 import A_Adiag_PolynomialParams_KpmEstimate
    F, Q, w = dense["F"], dense["Q"], dense["w"]
    Ad = torch.from_numpy(np.diag(F.Hd.numpy()).copy())
    bound = OOC2_KrylovAv_A_EstimateSpectrumBound(None, F)
    S, V = S_HeigvalCDSIHD_HeigvecCDSIHD(F, Ad, k=16, tol=1e-10, User_ChebyshevDegree=20, User_SpectrumBound=bound)
    assert np.max(np.abs(np.asarray(S.cpu()) - w[:16]) / w[:16]) < 1e-9
    for bad in (dict(User_SpectrumBound=None), dict(User_SpectrumBound=bound, User_WorkspaceSizeFactor=1),
                dict(User_SpectrumBound=bound, User_Q_HotellingDeflation=Q)):
        with pytest.raises(AssertionError, match="ABORTED"):
            S_HeigvalCDSIHD_HeigvecCDSIHD(F, Ad, k=16, **bad)
    lo, hi = 0.5 * (w[9] + w[10]), 0.5 * (w[80] + w[81])
    pol = polyfilter.OOC0_OptimizePolynomialParamsOnDegree(User_WantedInterval=(lo, hi),
                                                           User_SpectrumBound=(w[0] - 1e-3, w[-1] * 1.01),
                                                           User_MaximumDegree=3000)
    true = int(np.sum((w >= lo) & (w <= hi)))
    est = A_Adiag_PolynomialParams_KpmEstimate(F, Ad, User_PolynomialParams=pol, User_NumberKpmTrials=400)
    assert abs(est - true) <= 0.3 * true


class RankOneStore:
    """Host view of the rank-one store built by the oracle: cutoff lists and FP64
    entries {wx, wy, wz, col} with w = (x_j - x_i) / |x_j - x_i| (0 for the self
    entry), as the Galerkin bead operator reads them."""

    def __init__(self, X):
        from oracle import graph as og
        deg, rp, cl = og.neighbor_lists(X, 8.0)
        n = X.shape[0]
        rows = np.repeat(np.arange(n), np.diff(rp))
        d = X[cl] - X[rows]
        nrm = np.linalg.norm(d, axis=1)
        w = np.where(nrm[:, None] > 0, d / np.where(nrm > 0, nrm, 1.0)[:, None], 0.0)
        self.X = torch.from_numpy(X)
        self.rowptr = torch.from_numpy(np.asarray(rp, np.int64))
        self.cols = torch.from_numpy(np.asarray(cl, np.int32))
        self.ent64 = torch.from_numpy(np.c_[w, cl.astype(np.float64)])
        self.ent32 = None
        self.n_atoms, self.plus_i, self.device = n, 1.0, torch.device("cpu")
        self.shape = (3 * n, 3 * n)


def test_galerkin_bead_operator_and_start_on_cpu():
    """The Galerkin bead operator built from the store's w entries equals
    M^-1/2 P^T H P M^-1/2 of the oracle Hessian, and the Galerkin start's block
    V = P M^-1/2 Z is orthonormal with V^T H V carrying the operator's lowest
    non-rigid eigenvalues."""
    import scipy.sparse as sp
    from inching_b200 import synth
    from inching_b200.warmstart import GalerkinOperator, bead_model, galerkin_warm_start
    X = synth.globule(600, seed=8) / 10.0
    H = RankOneStore(X)
    A, Ad = oh.hessian_lower(X, 8.0, 1.0)
    Hd = oh.full_from_lower(A, Ad).toarray()
    _, bead = bead_model(H.X, 6.0)
    nb = int(bead.max()) + 1
    counts = torch.bincount(bead, minlength=nb)
    G = GalerkinOperator(H, bead, nb, counts)
    n = H.n_atoms
    bd = bead.numpy()
    P = sp.csr_matrix((np.ones(3 * n), (np.arange(3 * n), 3 * np.repeat(bd, 3) + np.tile([0, 1, 2], n))),
                      shape=(3 * n, 3 * nb))
    Mh = 1.0 / np.sqrt(np.repeat(counts.numpy(), 3).astype(float))
    S = (sp.diags(Mh) @ (P.T @ sp.csr_matrix(Hd) @ P) @ sp.diags(Mh)).toarray()
    assert np.abs(G.csr64.to_dense().numpy() - S).max() < 1e-12 * np.abs(S).max()
    V, info = galerkin_warm_start(H, 24, tol=1e-6, return_info=True)
    assert V.shape == (3 * n, 24) and info["beads"] == nb
    assert (V.t() @ V - torch.eye(24, dtype=V.dtype)).abs().max() < 1e-10
    theta = np.linalg.eigvalsh((V.t() @ torch.from_numpy(Hd) @ V).numpy())
    sigma = np.linalg.eigvalsh(S)[6:30]
    assert np.abs(theta - sigma).max() < 1e-6 * sigma[-1]
