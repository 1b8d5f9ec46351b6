"""Autotuner host logic on CPU: the fastest candidate is applied, the choice is
cached per (atoms, pairs, width class, precision, device), the row-tile layout
is tried only when the store has tiles, and the launch-shape hook of the C ABI
accepts the documented shapes and rejects others (no GPU call is involved)."""
import pytest
import torch

COST = {("pairs", 256, 5): 3.0, ("pairs", 256, 4): 2.0, ("pairs", 512, 2): 2.5, ("pairs", 1024, 1): 4.0,
        ("pairs", 0, 4): 1.5, ("tiles", 256, 5): 1.0}


class FakeStore:
    def __init__(self, tiles):
        self.n_atoms, self.nnz_blocks = 100, 900
        self.shape = (300, 300)
        self.device = torch.device("cpu")
        self.tiles = {} if tiles else None
        self.use_tiles = False
        self.calls = 0

    def matmul(self, X, out=None, prec=32):
        self.calls += 1
        out.copy_(X)
        return out


def test_autotuner_picks_fastest_and_caches(monkeypatch):
    from inching_b200 import autotune
    applied = []
    monkeypatch.setattr(autotune._native, "spmm_tune", lambda t, b: applied.append((t, b)))
    autotune._cache.clear()
    timed = []

    def timer(fn, reps):
        fn()
        cfg = (("tiles" if H.use_tiles else "pairs"),) + applied[-1]
        timed.append(cfg)
        return COST[cfg]

    H = FakeStore(tiles=False)
    best, table = autotune.tune_spmm(H, 64, timer=timer)
    assert best == ("pairs", 0, 4) and applied[-1] == (0, 4) and not H.use_tiles
    assert set(table) == {c for c in COST if c[0] == "pairs"} and len(timed) == 5 and H.calls == 5
    again = autotune.tune_spmm(H, 100, timer=timer)          # same width class (64): cached
    assert again[0] == best and len(timed) == 5 and applied[-1] == (0, 4)
    autotune.tune_spmm(H, 16, timer=timer)                   # another width class: timed again
    assert len(timed) == 10
    H = FakeStore(tiles=True)
    H.nnz_blocks = 901                                       # another store
    best, table = autotune.tune_spmm(H, 64, timer=timer)
    assert best == ("tiles", 256, 5) and H.use_tiles and applied[-1] == (256, 5) and len(table) == 6
    autotune._cache.clear()


def test_launch_shape_hook_accepts_documented_shapes_only():
    from inching_b200 import _native, autotune
    for t, b in ((256, 5), (512, 2), (1024, 1), (0, 4)):
        _native.spmm_tune(t, b)
    with pytest.raises(AssertionError):
        _native.spmm_tune(300, 5)
    autotune.reset()
    assert autotune._cache == {}
