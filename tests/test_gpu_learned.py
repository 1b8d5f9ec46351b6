"""Learned warm start: the hand-written forward/backward kernels against the CPU
oracle, the Hellmann-Feynman gradient and the weighted bead Hessian against
dense references, and what the trained network gains over the method without it.

Tolerances: network outputs and gradients in FP32 vs the FP64 oracle, relative
1e-4 (outputs) and 2e-3 (gradient norms per tensor); FP64 Hessian/gradients 1e-10."""
import os

import numpy as np
import pytest
import torch

from oracle import mpnn as om

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bead():
    from inching_b200 import graph, synth
    from inching_b200.hessian import HessianStore
    from inching_b200.learned import BeadGraph
    X = synth.globule(3000, seed=41) / 10.0
    Xd = torch.from_numpy(X).cuda()
    H = HessianStore(Xd, 8.0, 1.0, precisions=("f64",))
    return BeadGraph(Xd, H.rowptr, H.cols)


def _np(t):
    return t.detach().double().cpu().numpy()


def test_forward_backward_match_oracle(bead):
    from inching_b200.learned import WarmStartMPNN
    G = bead
    model = WarmStartMPNN(seed=3)
    # make the readout non-trivial so every layer carries gradient
    model.p["wo"].mul_(50.0)
    gamma, cache = model.forward(G)
    p = {k: _np(v) for k, v in model.p.items()}
    x, ef, src, dst = _np(G.x), _np(G.ef), G.src.long().cpu().numpy(), G.dst.long().cpu().numpy()
    gref, cref = om.forward(p, x, ef, src, dst, G.n)
    assert np.max(np.abs(_np(gamma) - gref) / gref) < 1e-4
    dgamma = torch.from_numpy(np.random.default_rng(0).standard_normal(G.E)).cuda()
    model.backward(G, cache, dgamma)
    gr = om.backward(p, x, ef, src, dst, G.n, cref, _np(dgamma))
    for name in p:
        a, b = _np(model.g[name]), gr[name]
        assert np.linalg.norm(a - b) <= 2e-3 * max(np.linalg.norm(b), 1e-8), name


def test_weighted_bead_hessian_and_eigen_gradient(bead):
    from inching_b200 import _native
    from inching_b200.hessian import HessianStore
    G = bead
    src, dst = G.src.long().cpu().numpy(), G.dst.long().cpu().numpy()
    # symmetric random spring constants
    key = np.minimum(src, dst) * G.n + np.maximum(src, dst)
    gam = 0.5 + (np.sin(key * 0.37) + 1.0)
    gam_t = torch.from_numpy(gam).cuda()
    Hb = HessianStore(G.pos, G.rc_nm * 10.0, 1.0, precisions=("f64",), graph_=(G.degree, G.rowptr, G.cols),
                      pair_weight=G.adjacency_weights(gam_t))
    Hd = om.bead_hessian(_np(G.pos), src, dst, gam)
    v = np.random.default_rng(2).standard_normal((Hd.shape[0], 3))
    y = Hb.matmul(torch.from_numpy(v).cuda().contiguous())
    assert np.abs(_np(y) - Hd @ v).max() < 1e-10 * np.abs(Hd).max() * 10
    w, V = np.linalg.eigh(Hd)
    c = np.random.default_rng(3).standard_normal(8)
    Vsel = np.ascontiguousarray(V[:, 6:14])
    out = torch.empty(G.E, dtype=torch.float64, device="cuda")
    _native.mp("hf_grad", G.pos, G.mp_rowptr, G.src, G.dst, torch.from_numpy(Vsel).cuda(), 8,
               torch.from_numpy(c).cuda(), G.E, out)
    ref = om.hf_grad(_np(G.pos), src, dst, Vsel, c)
    assert np.abs(_np(out) - ref).max() < 1e-10 * max(np.abs(ref).max(), 1.0)


def _bead_err(G, gam, lam_f):
    from inching_b200.learned import bead_modes
    lam, _ = bead_modes(G, gam, lam_f.shape[0])
    return float(torch.sqrt((((lam - lam_f) / lam_f) ** 2).mean()))


def test_trained_network_gain():
    """Train on six synthetic structures (60 epochs, a few seconds), then on two
    held-out structures compare the bead model's eigenvalue error with uniform
    springs and with the learned ones, and the fine block solver's iterations
    from a random start and from the learned start (which must pass its residual
    test against a random block)."""
    from inching_b200 import graph, synth
    from inching_b200.deflation import rigid_body_basis
    from inching_b200.hessian import HessianStore
    from inching_b200.learned import WarmStartMPNN, learned_warm_start, make_sample, train, training_structures
    from inching_b200.solvers.chfsi import chfsi
    samples = [make_sample(X, m=24) for X in training_structures(6, seed=11)]
    model = WarmStartMPNN(seed=1)
    hist = train(model, samples, epochs=60, lr=3e-3, verbose=False)
    assert hist[-1] < 0.3 * hist[0]
    held = [synth.touching_assembly([1500] * 4, seed=999) / 10.0, synth.globule(5000, seed=998) / 10.0]
    err_u, err_l = [], []
    for X in held:
        G, lam_f = make_sample(X, m=24)
        err_u.append(_bead_err(G, torch.ones(G.E, dtype=torch.float64, device="cuda"), lam_f))
        err_l.append(_bead_err(G, model.forward(G)[0], lam_f))
    assert np.mean(err_l) < 0.8 * np.mean(err_u)
    Xd = torch.from_numpy(held[0]).cuda()
    order, _ = graph.cuthill_mckee(Xd, 8.0)
    Xr = Xd[order]
    H = HessianStore(Xr, 8.0, 1.0)
    Q = rigid_body_basis(Xr)
    k, p = 48, 48 + 16
    _, _, i0 = chfsi(H, k, tol=1e-6, Q=Q, precision="mixed", return_info=True)
    X0, winfo = learned_warm_start(Xr, p, model, H.rowptr, H.cols, H=H, Q=Q, k=k, return_info=True)
    assert not winfo["fallback"]
    _, _, i1 = chfsi(H, k, tol=1e-6, Q=Q, precision="mixed", X0=X0, return_info=True)
    print(f"\nbead-model eigenvalue rms rel error on held-out: uniform {np.round(err_u, 3)}, "
          f"learned {np.round(err_l, 3)}; fine iterations random {i0['iterations']}, learned {i1['iterations']}; "
          f"median Ritz residual random {winfo['random_median_residual']:.3g}, "
          f"learned {winfo['warm_median_residual']:.3g}")
    assert i1["max_rel_residual"] <= 1.5e-6
    assert i1["iterations"] <= i0["iterations"]


def test_fallback_to_random_start():
    """A network whose spring constants are not finite falls back to the random
    block; the solve from it still converges."""
    from inching_b200 import synth
    from inching_b200.deflation import rigid_body_basis
    from inching_b200.hessian import HessianStore
    from inching_b200.learned import WarmStartMPNN, learned_warm_start
    from inching_b200.solvers.chfsi import chfsi
    Xr = torch.from_numpy(synth.globule(2000, seed=5) / 10.0).cuda()
    H = HessianStore(Xr, 8.0, 1.0)
    Q = rigid_body_basis(Xr)
    model = WarmStartMPNN(seed=0)
    model.flat.fill_(float("nan"))
    X0, info = learned_warm_start(Xr, 32, model, H.rowptr, H.cols, H=H, Q=Q, k=16, return_info=True)
    assert info["fallback"] and "warm_median_residual" not in info
    assert bool(torch.isfinite(X0).all())
    _, _, i = chfsi(H, 16, tol=1e-6, Q=Q, precision="mixed", X0=X0, return_info=True)
    assert i["converged"]


def test_pipeline_with_shipped_weights():
    """normal_modes(..., warm_start="learned") with the weights shipped in the
    package: passes the residual test and converges to tol with the same
    eigenvalues as the random start."""
    from inching_b200 import synth
    from inching_b200.pipeline import normal_modes_device
    Xd = torch.from_numpy(synth.touching_assembly([1500] * 4, seed=999) / 10.0).cuda()
    e0, _, i0 = normal_modes_device(Xd, 48, tol=1e-6)
    e1, _, i1 = normal_modes_device(Xd, 48, tol=1e-6, warm_start="learned")
    assert not i1["warm_start"]["fallback"]
    assert i1["max_rel_residual"] <= 1.5e-6
    assert i1["iterations"] <= i0["iterations"]
    assert float(((e1 - e0).abs() / e0).max()) < 1e-6


def test_learned_start_beats_uniform_bead_start_on_held_out():
    """What the trained network gains over the method without it: on a held-out
    20,000-atom assembly (not among the training structures), the fine block solver
    from the shipped network's bead start needs fewer iterations and fewer filter
    SpMMs than from the uniform bead model (measured on the B200: 6 / 120 against
    7 / 144), with the same eigenvalues."""
    from inching_b200 import graph, synth
    from inching_b200.deflation import rigid_body_basis
    from inching_b200.hessian import HessianStore
    from inching_b200.learned import WarmStartMPNN, learned_warm_start
    from inching_b200.solvers.chfsi import chfsi_lean, default_guard
    from inching_b200.warmstart import coarse_warm_start
    Xd = torch.from_numpy(synth.touching_assembly([5000] * 4, seed=77) / 10.0).cuda()
    order, _ = graph.cuthill_mckee(Xd, 8.0)
    Xr = Xd[order]
    H = HessianStore(Xr, 8.0, 1.0)
    Q = rigid_body_basis(Xr)
    k = 128
    p = k + default_guard(k)
    Xu = coarse_warm_start(Xr, p, wanted=k)
    eu, _, iu = chfsi_lean(H, k, tol=1e-6, Q=Q, precision="mixed", X0=Xu, return_info=True)
    Xl, w = learned_warm_start(Xr, p, WarmStartMPNN.load(), H.rowptr, H.cols, H=H, Q=Q, k=k, return_info=True)
    el, _, il = chfsi_lean(H, k, tol=1e-6, Q=Q, precision="mixed", X0=Xl, return_info=True)
    print(f"\nuniform beads: {iu['iterations']} iterations, {iu['n_spmm_filter']} filter SpMMs; "
          f"learned: {il['iterations']}, {il['n_spmm_filter']}")
    assert not w["fallback"]
    assert il["max_rel_residual"] <= 1.5e-6 and iu["max_rel_residual"] <= 1.5e-6
    assert il["iterations"] < iu["iterations"]
    assert il["n_spmm_filter"] < iu["n_spmm_filter"]
    assert float(((el - eu).abs() / eu).max()) < 1e-6


@pytest.mark.parametrize("M,N,K,ta,tb", [(300, 128, 137, False, False), (7800, 128, 263, False, False),
                                         (263, 128, 60000, True, False), (1, 128, 50000, False, False),
                                         (5000, 263, 128, False, True), (129, 1, 263, False, False)])
def test_dense_layer_kernel_matches_torch(M, N, K, ta, tb):
    """The network's dense-layer kernel (inch_mp_gemm) against a torch FP32 matmul of
    the same operands: forward (X W), weight gradient (X^T dY, long K with the
    deterministic split-K), input gradient (dY W^T), column sums, a single column;
    accumulating into C with beta = 1.  Tolerance 1e-5 of the largest output."""
    from inching_b200 import _native
    g = torch.Generator(device="cuda")
    g.manual_seed(M + N + K)
    A = torch.randn((K, M) if ta else (M, K), generator=g, device="cuda")
    B = torch.randn((N, K) if tb else (K, N), generator=g, device="cuda")
    Av = A.t() if ta else A
    Bv = B.t() if tb else B
    ref = Av @ Bv
    C = torch.empty((M, N), device="cuda")
    _native.mp_gemm(Av, Bv, C)
    scale = float(ref.abs().max())
    assert float((C - ref).abs().max()) <= 1e-5 * scale * max(1.0, K ** 0.5 / 10)
    C0 = torch.randn((M, N), generator=g, device="cuda")
    C1 = C0.clone()
    _native.mp_gemm(Av, Bv, C1, beta=1.0)
    assert float((C1 - (C0 + ref)).abs().max()) <= 1e-5 * (scale + float(C0.abs().max())) * max(1.0, K ** 0.5 / 10)
    # deterministic: the same call twice gives the same bits
    C2 = torch.empty((M, N), device="cuda")
    _native.mp_gemm(Av, Bv, C2)
    assert torch.equal(C, C2)
