"""Row-block pieces on one GPU: the store rows a rank builds (columns rebased to
its halo range, empty halo rows) give the full store's product rows, and the
row-block solver on a single rank (no process group) finds the pipeline's
eigenvalues."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_store_rows_match_full_store_and_single_rank_solve():
    from inching_b200 import _native, graph, synth
    from inching_b200.hessian import HessianStore
    from inching_b200.pipeline import normal_modes_device
    from inching_b200.rowblock import StoreRows, halo_ranges, row_partition, rowblock_normal_modes
    X = torch.from_numpy(synth.globule(3000, seed=4) / 10.0).cuda()
    order, _ = graph.cuthill_mckee(X, 8.0)
    Xr = X[order].contiguous()
    _, rp, cl = _native.neighbor_lists(Xr, 0.8)
    H = HessianStore(Xr, 8.0, 1.0)
    parts = row_partition(rp, 3)
    ranges = halo_ranges(rp, cl, parts)
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    V = torch.randn((Xr.shape[0] * 3, 16), generator=g, dtype=torch.float64, device="cuda")
    for prec, dt, tol in ((64, torch.float64, 1e-13), (32, torch.float32, 1e-5)):
        Vp = V.to(dt).contiguous()
        full = H.matmul(Vp, prec=prec)
        scale = float(full.abs().max())
        for (a, b), (lo, hi) in zip(parts, ranges):
            loc = StoreRows(Xr, 8.0, 1.0, rp, cl, a, b, lo, hi)
            y = loc.local_matmul(Vp[3 * lo:3 * hi].contiguous(), prec)
            assert y.shape == (3 * (b - a), 16)
            assert float((y - full[3 * a:3 * b]).abs().max()) <= tol * scale
    e0, m0, _ = normal_modes_device(X, 24, tol=1e-9, precision="f64")
    e1, m1, info = rowblock_normal_modes(X, 24, tol=1e-9, precision="f64")
    assert info["converged"] and info["parts"] == [(0, Xr.shape[0])]
    assert float(((e1 - e0).abs() / e0).max()) < 1e-9
    assert m1.shape == m0.shape
    # same modes up to sign (the spectrum of this globule has no degenerate pair among the 24)
    ov = torch.einsum("kna,kna->k", m0, m1) / (m0.norm(dim=(1, 2)) * m1.norm(dim=(1, 2)))
    assert float((ov.abs() - 1).abs().max()) < 1e-6
