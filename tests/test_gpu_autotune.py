"""Every launch choice the autotuner can make gives the same product (the
default pair kernel's, within FP32 / FP64 rounding of a different summation
order), and tune_spmm records its choice on the store, which re-applies it."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def store():
    from inching_b200 import graph, synth
    from inching_b200.hessian import HessianStore
    X = synth.globule(3000, seed=8) / 10.0
    order, _ = graph.cuthill_mckee(X, 8.0)
    return HessianStore(X[order.cpu().numpy()], 8.0, plus_i=1.0, tiles=True)


@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("b", [64, 200])
def test_every_candidate_gives_the_default_product(store, prec, b):
    from inching_b200 import autotune
    H = store
    dt = torch.float32 if prec == 32 else torch.float64
    g = torch.Generator(device="cuda")
    g.manual_seed(b)
    X = torch.randn((H.shape[0], b), generator=g, dtype=torch.float64, device="cuda").to(dt)
    try:
        autotune.apply_config(H, ("pairs", 256, 5, 1))
        ref = H.matmul(X, prec=prec).double()
        scale = float(ref.abs().max())
        tol = 2e-6 if prec == 32 else 1e-13
        for cfg in autotune.CANDIDATES:
            autotune.apply_config(H, cfg)
            Y = H.matmul(X, prec=prec).double()
            assert float((Y - ref).abs().max()) <= tol * scale, cfg
    finally:
        autotune.reset()
        H.use_tiles = True


def test_tune_records_choice_on_store(store):
    from inching_b200 import autotune
    H = store
    try:
        best, table = autotune.tune_spmm(H, 64, prec=32)
        assert best in autotune.CANDIDATES and best in table
        assert H.spmm_cfg[(32, 64)] == best
        assert all(ms > 0 for ms in table.values())
    finally:
        autotune.reset()
        H.spmm_cfg.clear()
        H.use_tiles = True
